// stage_d4_mix.cu -- stage-kernel instantiations for MCV4, split precision:
// the tile shapes (cells x cells, threads, CTAs per SM the registers must allow,
// sweep style (0: per-cell items, n: walks of n cells), TMA-staged persistent
// form) the autotuner chooses from; split-precision sweeps run on packed FP32
// pairs.
// the last entry's option bits (OPT 3) balance the sweep walks and form
// each loaded column's linear references once per work item.
#include "mcv_stage.cuh"

namespace mcv {

const StageLauncher *stage_launchers_d4_mix(int *count) {
  static const StageLauncher table[] = {
    StageConfig<4, 8, 8, 320, 2, true, 0>::make(),
    StageConfig<4, 8, 8, 320, 3, true, 0>::make(),
    StageConfig<4, 8, 8, 256, 3, true, 0>::make(),
    StageConfig<4, 8, 8, 320, 2, true, 2>::make(),
    StageConfig<4, 8, 8, 256, 2, true, 0, true>::make(),
    StageConfig<4, 8, 8, 320, 2, true, 0, true>::make(),
    StageConfig<4, 8, 8, 320, 2, true, 2, true, 3>::make()};
  *count = (int)(sizeof(table) / sizeof(table[0]));
  return table;
}

}  // namespace mcv
