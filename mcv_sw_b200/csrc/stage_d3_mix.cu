// stage_d3_mix.cu -- stage-kernel instantiations for MCV3, split precision:
// the tile shapes (cells x cells, threads, sweep style) the autotuner chooses from.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d3_mix(int *count) {
  static const StageLauncher table[] = {
    StageConfig<3, 12, 12, 320, true, false>::make(),
    StageConfig<3, 16, 12, 448, true, false>::make(),
    StageConfig<3, 16, 16, 512, true, false>::make(),
    StageConfig<3, 12, 12, 160, true, true>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
