// stage_d4_f64.cu -- stage-kernel instantiations for MCV4, FP64:
// the tile shapes (cells x cells, threads, CTAs per SM the registers must allow,
// sweep style (0: per-cell items, n: walks of n cells), TMA-staged persistent
// form) the autotuner chooses from.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d4_f64(int *count) {
  static const StageLauncher table[] = {
    StageConfig<4, 8, 8, 320, 2, false, 0>::make(),
    StageConfig<4, 6, 6, 256, 3, false, 0>::make(),
    StageConfig<4, 6, 6, 256, 3, false, 2>::make(),
    StageConfig<4, 6, 6, 256, 3, false, 3>::make(),
    StageConfig<4, 8, 8, 320, 2, false, 2>::make(),
    StageConfig<4, 6, 6, 256, 2, false, 0, true>::make(),
    StageConfig<4, 8, 8, 320, 1, false, 0, true>::make(),
    StageConfig<4, 8, 8, 640, 1, false, 2, true>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
