// stage_d4_f64.cu -- stage-kernel instantiations for MCV4, FP64:
// the tile shapes (cells x cells, threads, CTAs per SM the registers must allow,
// sweep style, TMA-staged persistent form) the autotuner chooses from.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d4_f64(int *count) {
  static const StageLauncher table[] = {
    StageConfig<4, 8, 8, 320, 2, false, false>::make(),
    StageConfig<4, 6, 6, 256, 3, false, false>::make(),
    StageConfig<4, 8, 8, 256, 2, false, false>::make(),
    StageConfig<4, 6, 6, 128, 3, false, true>::make(),
    StageConfig<4, 6, 6, 256, 2, false, false, true>::make(),
    StageConfig<4, 8, 8, 320, 1, false, false, true>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
