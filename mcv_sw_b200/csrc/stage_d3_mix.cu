// stage_d3_mix.cu -- stage-kernel instantiations for MCV3, split precision:
// the tile shapes (cells x cells, threads, CTAs per SM the registers must allow,
// sweep style, TMA-staged persistent form) the autotuner chooses from.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d3_mix(int *count) {
  static const StageLauncher table[] = {
    StageConfig<3, 12, 12, 320, 2, true, false>::make(),
    StageConfig<3, 12, 12, 320, 3, true, false>::make(),
    StageConfig<3, 12, 12, 256, 4, true, false>::make(),
    StageConfig<3, 16, 12, 448, 2, true, false>::make(),
    StageConfig<3, 12, 12, 160, 1, true, true>::make(),
    StageConfig<3, 12, 12, 320, 2, true, false, true>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
