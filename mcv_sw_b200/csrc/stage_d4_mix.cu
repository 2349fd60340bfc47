// stage_d4_mix.cu -- stage-kernel instantiations for MCV4, split precision:
// the tile shapes (cells x cells, threads, sweep style) the autotuner chooses from.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d4_mix(int *count) {
  static const StageLauncher table[] = {
    StageConfig<4, 8, 8, 320, true, false>::make(),
    StageConfig<4, 8, 8, 256, true, false>::make(),
    StageConfig<4, 12, 8, 448, true, false>::make(),
    StageConfig<4, 12, 12, 224, true, true>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
