// stage_d3_f64.cu -- stage-kernel instantiations for MCV3, FP64:
// the tile shapes (cells x cells, threads, CTAs per SM the registers must allow,
// sweep style (0: per-cell items, n: walks of n cells), TMA-staged persistent
// form) the autotuner chooses from.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d3_f64(int *count) {
  static const StageLauncher table[] = {
    StageConfig<3, 12, 12, 320, 2, false, 0>::make(),
    StageConfig<3, 8, 8, 224, 4, false, 0>::make(),
    StageConfig<3, 8, 8, 160, 4, false, 0>::make(),
    StageConfig<3, 16, 8, 384, 2, false, 0>::make(),
    StageConfig<3, 12, 12, 320, 2, false, 2>::make(),
    StageConfig<3, 8, 8, 224, 4, false, 2>::make(),
    StageConfig<3, 8, 8, 224, 2, false, 0, true>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
