// stage_d3_mix.cu -- stage-kernel instantiations for MCV3, split precision:
// the tile shapes (cells x cells, threads, CTAs per SM the registers must allow,
// sweep style (0: per-cell items, n: walks of n cells), TMA-staged persistent
// form) the autotuner chooses from; split-precision sweeps run on packed FP32
// pairs.
// the TMA walk entries form each loaded column's linear references once per
// work item (OPT bit 2); the walks of 3 cells also balance the sweep walks (bit 1).
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d3_mix(int *count) {
  static const StageLauncher table[] = {
    StageConfig<3, 12, 12, 320, 2, true, 0>::make(),
    StageConfig<3, 12, 12, 320, 3, true, 0>::make(),
    StageConfig<3, 12, 12, 256, 3, true, 0>::make(),
    StageConfig<3, 12, 12, 320, 2, true, 2>::make(),
    StageConfig<3, 16, 12, 448, 2, true, 0>::make(),
    StageConfig<3, 12, 12, 320, 2, true, 0, true>::make(),
    StageConfig<3, 12, 12, 320, 2, true, 2, true, 2>::make(),
    StageConfig<3, 12, 12, 320, 2, true, 3, true, 3>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
