// mcv_gpu.cu -- C ABI (include/mcv_gpu.h) over the sm_100a kernels.
//
// A handle holds one grid (order, Nc) and `members` states, all resident in
// HBM.  One RK step is 2 * stages kernel launches (fused stage K1, halo K2),
// captured into a CUDA graph and replayed per step.  The stage kernel's tile
// shape is chosen per handle by timing every candidate shape on the handle's
// own grid before the first step (the autotuner).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mcv_gpu.h"
#include "mcv_halo.cuh"
#include "mcv_internal.h"

namespace mcv {

static thread_local std::string g_last_error;

int fail(int code, const char *msg) {
  g_last_error = msg;
  return code;
}

static int cuda_fail(cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  g_last_error = m;
  return (e == cudaErrorMemoryAllocation) ? MCV_ERR_NOMEM : MCV_ERR_CUDA;
}

#define MCV_CUDA(call, what)                           \
  do {                                                 \
    cudaError_t _e = (call);                           \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

const StageLauncher *stage_launchers_d3_f64(int *count);
const StageLauncher *stage_launchers_d3_mix(int *count);
const StageLauncher *stage_launchers_d4_f64(int *count);
const StageLauncher *stage_launchers_d4_mix(int *count);

const StageLauncher *stage_launchers(int order, bool mixed, int *count) {
  if (order == 3) return mixed ? stage_launchers_d3_mix(count) : stage_launchers_d3_f64(count);
  return mixed ? stage_launchers_d4_mix(count) : stage_launchers_d4_f64(count);
}

// Cube connectivity from CubedSphereFillHalo (src/ghost_mod.f90:104-146):
// {neighbour panel, neighbour edge, reversed}, panels 0-based, edges W E S N.
static const int kLinks[6][4][3] = {
    {{3, 1, 0}, {1, 0, 0}, {5, 3, 0}, {4, 2, 0}},  // panel 1
    {{0, 1, 0}, {2, 0, 0}, {5, 1, 1}, {4, 1, 0}},  // panel 2
    {{1, 1, 0}, {3, 0, 0}, {5, 2, 1}, {4, 3, 1}},  // panel 3
    {{2, 1, 0}, {0, 0, 0}, {5, 0, 0}, {4, 0, 1}},  // panel 4
    {{3, 3, 1}, {1, 3, 0}, {0, 3, 0}, {2, 3, 1}},  // panel 5
    {{3, 2, 0}, {1, 2, 1}, {2, 2, 1}, {0, 2, 0}},  // panel 6
};
// The eight cube vertices in unify_bdy_field's term order
// (src/spatial_operators_mod.F90:347-386): (panel, corner) x 3, corners SW SE NW NE.
static const int kVertices[8][3][2] = {
    {{0, 2}, {3, 3}, {4, 0}},  // (1,4,5)
    {{0, 3}, {1, 2}, {4, 1}},  // (1,2,5)
    {{0, 0}, {3, 1}, {5, 2}},  // (1,4,6)
    {{0, 1}, {1, 0}, {5, 3}},  // (1,2,6)
    {{2, 2}, {1, 3}, {4, 3}},  // (2,3,5)
    {{2, 3}, {3, 2}, {4, 2}},  // (3,4,5)
    {{1, 1}, {2, 0}, {5, 1}},  // (2,3,6)
    {{2, 1}, {3, 0}, {5, 0}},  // (3,4,6)
};

static int upload_tables() {
  EdgeLink links[6][4];
  for (int p = 0; p < 6; ++p)
    for (int e = 0; e < 4; ++e)
      links[p][e] = EdgeLink{(int8_t)kLinks[p][e][0], (int8_t)kLinks[p][e][1], (int8_t)kLinks[p][e][2], 0};
  VertexRef verts[6][4];
  std::memset(verts, 0xff, sizeof(verts));
  for (int v = 0; v < 8; ++v)
    for (int t = 0; t < 3; ++t) {
      VertexRef r;
      for (int s = 0; s < 3; ++s) {
        r.panel[s] = (int8_t)kVertices[v][s][0];
        r.corner[s] = (int8_t)kVertices[v][s][1];
      }
      verts[kVertices[v][t][0]][kVertices[v][t][1]] = r;
    }
  MCV_CUDA(cudaMemcpyToSymbol(c_links, links, sizeof(links)), "upload edge links");
  MCV_CUDA(cudaMemcpyToSymbol(c_vertex, verts, sizeof(verts)), "upload vertex table");
  return MCV_OK;
}

constexpr double kOmega = 7.292E-5;  // constants_mod.F90:18
constexpr int kPartialBlocks = 296;

}  // namespace mcv

using namespace mcv;

struct mcv_handle {
  int order = 0, nc = 0, scheme = 0, precision = 0, members = 0;
  bool mixed = false;
  double dt = 0, radius = 0;
  GridDesc g{};
  int H = 0, npx = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  // device memory (one allocation)
  void *pool = nullptr;
  size_t pool_bytes = 0;
  // FP64 policy: state Y, stage buffers A, B, RK4 accumulator
  double *Y[3]{}, *A[3]{}, *B[3]{}, *acc[3]{};
  // split precision: FP64 state ping-pong S[cur], S[1-cur]; FP32 increments DA, DB
  double *S[2][3]{};
  int cur = 0;             // buffer the next step reads
  std::vector<int> mcur;   // buffer holding each member (members left out of steps keep theirs)
  float *DA[3]{}, *DB[3]{}, *facc[3]{};
  float *phis32 = nullptr;
  float4 *bnd32 = nullptr;
  double4 *met1d = nullptr;
  double *phibar = nullptr;
  double *prec = nullptr;  // TMA form: per (member, panel, tile) linear references of a step's first stage
  std::vector<double> phibar_host;
  // shared
  double *sqrtG = nullptr, *ig11 = nullptr, *ig12 = nullptr, *ig22 = nullptr, *fcor = nullptr, *phis = nullptr;
  double4 *bnd = nullptr, *Mtab = nullptr, *Ntab = nullptr;
  int *giref = nullptr;
  double2 *gcoef = nullptr;
  double4 *partial = nullptr;
  double dx2 = 0, dx3 = 0;
  bool geometry_set = false;
  std::vector<char> member_set;
  std::vector<long long> steps_done;
  // members the step advances: device list [n_active] read by both kernels
  int *active = nullptr;
  std::vector<int> active_host;
  int n_active = 0;
  // active_host[k] == k for every k: the kernels take the slot as the member
  // index without reading the list (the step graphs bake this in)
  bool active_ident = true;
  int *flags = nullptr;  // non-finite flags [members]
  int *err = nullptr;    // stage-kernel error flag (TMA staging timed out)
  double *stage = nullptr;  // one FP64 field in the host's dense layout (PCIe copies land here)
  double *area = nullptr;   // areaCell of one panel [nc][nc] (the error norms' weights)
  int nsm = 0;           // SMs of the device
  std::vector<int> bps;  // resident CTAs per SM of each candidate
  int launch_err = 0;    // status of the last stage launch (tensor-map encoding)
  std::vector<double> sqrtG_host;  // padded Fortran layout, for phiG on download
  // stage kernel chosen by the autotuner
  const StageLauncher *cands = nullptr;
  int ncands = 0, choice = -1;
  std::vector<float> tune_ms;
  cudaGraphExec_t graph_exec[2]{};
};

namespace {

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

void grid_desc(int order, int nc, GridDesc &g, int &H, int &npx) {
  H = order - 1;
  g.n = nc * (order - 1) + 1;
  g.np = g.n + 2 * H;
  npx = g.np;
  g.P = (int)align_up((size_t)g.np, 16);
  g.Nc = nc;
  g.plane = (long long)g.np * g.P;
  g.mstride = 6 * g.plane;
}

// Offsets of every device array inside the handle's single allocation.
struct Layout {
  size_t total = 0;
  size_t f64_state[9]{}, f64_acc[3]{}, mix_state[6]{}, mix_inc[6]{}, mix_acc[3]{};
  size_t metric[5]{}, phis = 0, phis32 = 0, bnd = 0, bnd32 = 0, M = 0, N = 0, iref = 0, coef = 0, partial = 0,
         met1d = 0, phibar = 0, active = 0, flags = 0, err = 0, stage = 0, prec = 0, area = 0;
};

Layout make_layout(const GridDesc &g, int H, int scheme, int precision, int members) {
  Layout L;
  const size_t f64 = (size_t)g.mstride * sizeof(double) * members;  // one FP64 padded field, all members
  const size_t f32 = (size_t)g.mstride * sizeof(float) * members;
  const size_t plane6 = (size_t)g.mstride * sizeof(double);
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  const bool rk4 = scheme == MCV_RK4;
  if (precision == MCV_FP64) {
    for (int k = 0; k < 9; ++k) L.f64_state[k] = take(f64);
    if (rk4)
      for (int k = 0; k < 3; ++k) L.f64_acc[k] = take(f64);
  } else {
    for (int k = 0; k < 6; ++k) L.mix_state[k] = take(f64);
    for (int k = 0; k < 6; ++k) L.mix_inc[k] = take(f32);
    if (rk4)
      for (int k = 0; k < 3; ++k) L.mix_acc[k] = take(f32);
    L.phis32 = take(f32);
    L.bnd32 = take(sizeof(float4) * 24 * (size_t)g.n * members);
    L.met1d = take(sizeof(double4) * (size_t)g.np);
    L.phibar = take(sizeof(double) * members);
    // 96-byte linear-reference records for the most tiles any candidate shape makes
    int ncand = 0, most = 0;
    const StageLauncher *cands = stage_launchers(H + 1, true, &ncand);
    for (int c = 0; c < ncand; ++c)
      most = std::max(most, ((g.Nc + cands[c].CX - 1) / cands[c].CX) * ((g.Nc + cands[c].CY - 1) / cands[c].CY));
    L.prec = take((size_t)96 * 6 * most * members);
  }
  for (int k = 0; k < 5; ++k) L.metric[k] = take(plane6);
  L.phis = take(f64);
  L.bnd = take(sizeof(double4) * 24 * (size_t)g.n * members);
  L.M = take(sizeof(double4) * 24 * (size_t)(H + 1) * g.n);
  L.N = take(sizeof(double4) * 24 * (size_t)(H + 1) * g.n);
  L.iref = take(sizeof(int) * (size_t)H * g.n);
  L.coef = take(sizeof(double2) * (size_t)H * g.n);
  L.partial = take(sizeof(double4) * kPartialBlocks);
  L.active = take(sizeof(int) * (size_t)members);
  L.flags = take(sizeof(int) * (size_t)members);
  L.err = take(sizeof(int));
  L.stage = take(sizeof(double) * 6 * (size_t)g.np * g.np);  // one dense host-layout FP64 field
  L.area = take(sizeof(double) * (size_t)g.Nc * g.Nc);         // areaCell of one panel
  L.total = off;
  return L;
}

// Rows of `cols` elements between a dense layout (pitch cols) and the pitched
// device layout: one thread per element, one block row per grid row.
__global__ void repack_kernel(double *dst, const double *src, int cols, int dpitch, int spitch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const long long r = blockIdx.y;
  if (c < cols) dst[r * dpitch + c] = src[r * spitch + c];
}

// Copy a host array in the reference's padded Fortran layout (npx*npx*6,
// contiguous) into the pitched device layout.  FP64 fields cross PCIe as one
// contiguous copy into the dense staging field and are repacked on the device
// (a pitched PCIe copy of ~6 KB rows ran at 37 GB/s, a contiguous one at 55).
int upload_padded(mcv_handle *h, void *dst, const void *src, size_t elem) {
  const size_t row = (size_t)h->npx * elem;
  const int rows = h->npx * 6;
  if (elem == sizeof(double) && h->stage && rows <= 65535) {
    MCV_CUDA(cudaMemcpyAsync(h->stage, src, row * rows, cudaMemcpyHostToDevice, h->stream), "upload field");
    repack_kernel<<<dim3((h->npx + 255) / 256, rows), 256, 0, h->stream>>>((double *)dst, h->stage, h->npx, h->g.P,
                                                                            h->npx);
    MCV_CUDA(cudaGetLastError(), "repack field");
    return MCV_OK;
  }
  MCV_CUDA(cudaMemcpy2DAsync(dst, (size_t)h->g.P * elem, src, row, row, (size_t)rows, cudaMemcpyHostToDevice,
                             h->stream),
           "upload field");
  return MCV_OK;
}

int download_padded(mcv_handle *h, double *dst, const double *src) {
  const size_t row = (size_t)h->npx * sizeof(double);
  const int rows = h->npx * 6;
  if (h->stage && rows <= 65535) {
    repack_kernel<<<dim3((h->npx + 255) / 256, rows), 256, 0, h->stream>>>(h->stage, src, h->npx, h->npx, h->g.P);
    MCV_CUDA(cudaGetLastError(), "repack field");
    MCV_CUDA(cudaMemcpyAsync(dst, h->stage, row * rows, cudaMemcpyDeviceToHost, h->stream), "download field");
    return MCV_OK;
  }
  MCV_CUDA(cudaMemcpy2DAsync(dst, row, src, (size_t)h->g.P * sizeof(double), row, (size_t)rows,
                             cudaMemcpyDeviceToHost, h->stream),
           "download field");
  return MCV_OK;
}

int num_stages(const mcv_handle *h) { return h->scheme == MCV_RK3_TVD ? 3 : 4; }

// Stage kind of stage s of the handle's scheme.
int stage_kind(const mcv_handle *h, int s) { return (h->scheme == MCV_RK3_TVD ? RK3_S1 : RK4_S1) + s; }

// Stage arguments of stage s of one RK step.  FP64: the buffer sequence of
// RK3_TVD / RK4 (src/time_scheme_mod.F90:13-69) with the last stage writing Y
// in place.  Split precision: stages carry FP32 increments over the FP64 state
// S[c]; the last stage writes S[1-c].
StageArgs stage_args(mcv_handle *h, int s, int c) {
  StageArgs a{};
  a.sqrtG = h->sqrtG; a.ig11 = h->ig11; a.ig12 = h->ig12; a.ig22 = h->ig22; a.fcor = h->fcor;
  a.phis = h->phis;
  a.bnd = h->bnd;
  a.active = h->active;
  a.ident = h->active_ident ? 1 : 0;
  a.err = h->err;
  const double dt = h->dt;
  const int kind = stage_kind(h, s);
  if (!h->mixed) {
    a.aU = h->acc[0]; a.aV = h->acc[1]; a.aP = h->acc[2];
    double *const *in, *const *out;
    double inc;
    switch (kind) {
      case RK3_S1: in = h->Y; out = h->A; inc = dt; break;
      case RK3_S2: in = h->A; out = h->B; inc = 0.25 * dt; break;
      case RK3_S3: in = h->B; out = h->Y; inc = 2. / 3. * dt; break;
      case RK4_S1: in = h->Y; out = h->A; inc = 0.5 * dt; break;
      case RK4_S2: in = h->A; out = h->B; inc = 0.5 * dt; break;
      case RK4_S3: in = h->B; out = h->A; inc = dt; break;
      default: in = h->A; out = h->Y; inc = dt; break;
    }
    a.us = in[0]; a.vs = in[1]; a.ps = in[2];
    a.u0 = h->Y[0]; a.v0 = h->Y[1]; a.p0 = h->Y[2];
    a.uo = out[0]; a.vo = out[1]; a.po = out[2];
    a.inc = inc;
    return a;
  }
  double *const *Y = h->S[c], *const *Yn = h->S[1 - c];
  a.yu = Y[0]; a.yv = Y[1]; a.yp = Y[2];
  a.uo = Yn[0]; a.vo = Yn[1]; a.po = Yn[2];
  a.fU = h->facc[0]; a.fV = h->facc[1]; a.fP = h->facc[2];
  a.phis32 = h->phis32; a.met1d = h->met1d; a.phibar = h->phibar; a.bnd32 = h->bnd32; a.prec = h->prec;
  a.two_omega = 2. * kOmega;
  a.r2 = h->radius * h->radius;
  float *const *din = nullptr, *const *dout = nullptr;
  float wd = 0.f, wt = 0.f;
  switch (kind) {
    case RK3_S1: dout = h->DA; wt = (float)dt; break;
    case RK3_S2: din = h->DA; dout = h->DB; wd = 0.25f; wt = (float)(0.25 * dt); break;
    case RK3_S3: din = h->DB; wd = (float)(2. / 3.); wt = (float)(2. / 3. * dt); break;
    case RK4_S1: dout = h->DA; wt = (float)(0.5 * dt); break;
    case RK4_S2: din = h->DA; dout = h->DB; wt = (float)(0.5 * dt); break;
    case RK4_S3: din = h->DB; dout = h->DA; wt = (float)dt; break;
    default: din = h->DA; wt = (float)dt; break;
  }
  if (din) { a.du = din[0]; a.dv = din[1]; a.dp = din[2]; }
  if (dout) { a.eu = dout[0]; a.ev = dout[1]; a.ep = dout[2]; }
  a.wd = wd;
  a.wt = wt;
  return a;
}

HaloArgs halo_args(mcv_handle *h, int s, int c) {
  HaloArgs a{};
  a.bnd = h->bnd;
  a.Mtab = h->Mtab;
  a.Ntab = h->Ntab;
  a.giref = h->giref;
  a.gcoef = h->gcoef;
  a.dx = h->g.dx;
  a.dx2 = h->dx2;
  a.dx3 = h->dx3;
  a.rdx = 1. / h->g.dx;
  a.rdx2 = 1. / h->dx2;
  a.r2dx3 = 1. / (2. * h->dx3);
  a.members = h->n_active;
  a.active = h->active;
  a.ident = h->active_ident ? 1 : 0;
  const int kind = stage_kind(h, s);
  if (!h->mixed) {
    double *const *out = (kind == RK3_S1 || kind == RK4_S1 || kind == RK4_S3) ? h->A
                         : (kind == RK3_S2 || kind == RK4_S2)                  ? h->B
                                                                               : h->Y;
    a.u = out[0]; a.v = out[1]; a.phi = out[2];
    return a;
  }
  if (last_stage(kind)) {
    a.u = h->S[1 - c][0]; a.v = h->S[1 - c][1]; a.phi = h->S[1 - c][2];
    return a;
  }
  a.u = h->S[c][0]; a.v = h->S[c][1]; a.phi = h->S[c][2];
  float *const *d = (kind == RK3_S1 || kind == RK4_S1 || kind == RK4_S3) ? h->DA : h->DB;
  a.du = d[0]; a.dv = d[1]; a.dp = d[2];
  a.bnd32 = h->bnd32;
  return a;
}

// The halo kernel of stage s over `count` handles (one order and arithmetic)
// with buffer parities curs, one launch.
template <int NB>
void launch_halo_batch(mcv_handle *const *hs, const int *curs, int count, int s, cudaStream_t st) {
  HaloBatch<NB> b;
  std::memset(&b, 0, sizeof(b));
  int slots = 0, nmax = 0;
  for (int k = 0; k < count; ++k) {
    mcv_handle *h = hs[k];
    b.g[k] = h->g;
    b.a[k] = halo_args(h, s, curs[k]);
    b.first[k] = slots;
    slots += h->n_active;
    nmax = std::max(nmax, h->g.n);
  }
  b.first[count] = slots;
  b.ngrids = count;
  const bool mixed_inc = hs[0]->mixed && !last_stage(stage_kind(hs[0], s));
  // x: segments of kHaloSeg positions along an edge; y: 6 panels x 4 edges;
  // z: grids' active members.  A block holds the segment's H + 1 lines.
  const int block = kHaloSeg * (hs[0]->H + 1);
  const dim3 grid((unsigned)((nmax + kHaloSeg - 1) / kHaloSeg), 24u, (unsigned)slots);
  // programmatic stream serialization: the blocks may become resident during
  // the stage kernel's last items and wait there (griddepcontrol.wait)
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(block);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (hs[0]->order == 3) {
    if (mixed_inc) cudaLaunchKernelEx(&cfg, halo_kernel<3, true, NB>, b);
    else cudaLaunchKernelEx(&cfg, halo_kernel<3, false, NB>, b);
  } else {
    if (mixed_inc) cudaLaunchKernelEx(&cfg, halo_kernel<4, true, NB>, b);
    else cudaLaunchKernelEx(&cfg, halo_kernel<4, false, NB>, b);
  }
}

void launch_halo(mcv_handle *h, int s, int c) { launch_halo_batch<1>(&h, &c, 1, s, h->stream); }

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return (PFN_cuTensorMapEncodeTiled_v12000)p;
  }();
  return fn;
}

// Tensor map of one padded field seen as a 2-D array [rows][P] (rows = all
// panels of all members, or of the one metric plane), box [box_y][box_x].
int encode_field(CUtensorMap *m, const void *base, bool f32, const GridDesc &g, long long rows, int box_x,
                 int box_y) {
  auto fn = encode_fn();
  if (!fn) return fail(MCV_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
  const cuuint64_t dims[2] = {(cuuint64_t)g.P, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)g.P * (f32 ? 4u : 8u)};
  const cuuint32_t box[2] = {(cuuint32_t)box_x, (cuuint32_t)box_y};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = fn(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                        const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(MCV_ERR_CUDA, "tensor map encoding failed");
  return MCV_OK;
}

// Tensor maps of the fields a TMA-form stage launch stages (the kernel's order).
int stage_maps(mcv_handle *h, const StageLauncher &L, const StageArgs &a, int kind, TileMaps &tm) {
  const long long per_member = (long long)h->members * 6 * h->g.np, plane = 6LL * h->g.np;
  const int bx = L.box_x, by = L.box_y;
  int rc;
  if (!h->mixed) {
    const double *f[8] = {a.us, a.vs, a.ps, a.phis, a.sqrtG, a.ig11, a.ig12, a.ig22};
    for (int k = 0; k < 8; ++k)
      if ((rc = encode_field(&tm.f[k], f[k], false, h->g, k < 4 ? per_member : plane, bx, by))) return rc;
    return MCV_OK;
  }
  const double *f64[3] = {a.yu, a.yv, a.yp};
  for (int k = 0; k < 3; ++k)
    if ((rc = encode_field(&tm.f[k], f64[k], false, h->g, per_member, bx, by))) return rc;
  if ((rc = encode_field(&tm.f[3], a.phis32, true, h->g, per_member, bx, by))) return rc;
  if (!first_stage(kind)) {
    const float *f32[3] = {a.du, a.dv, a.dp};
    for (int k = 0; k < 3; ++k)
      if ((rc = encode_field(&tm.f[4 + k], f32[k], true, h->g, per_member, bx, by))) return rc;
  }
  return MCV_OK;
}

// Grid k of a stage launch: the handle's grid descriptor with the candidate's
// tiles, its stage arguments, tensor maps and work items (edge-free ones first).
template <int NB>
int add_grid(StageBatch<NB> &b, int k, mcv_handle *h, const StageLauncher &L, int s, int c) {
  GridDesc g = h->g;
  g.tiles_x = (h->nc + L.CX - 1) / L.CX;
  g.tiles_y = (h->nc + L.CY - 1) / L.CY;
  b.g[k] = g;
  b.a[k] = stage_args(h, s, c);
  b.slots[k] = h->n_active;
  TileMaps &tm = b.tm[k];
  std::memset(&tm, 0, sizeof(tm));
  tm.total = g.tiles_x * g.tiles_y * 6 * h->n_active;  // work items (tile, panel, member)
  if (L.tma)
    if (int rc = stage_maps(h, L, b.a[k], stage_kind(h, s), tm)) return rc;
  return MCV_OK;
}

// Item ranges of a batch of `n` grids: every grid's edge-free items, then
// every grid's edge items.
template <int NB>
void number_items(StageBatch<NB> &b, int n) {
  b.ngrids = n;
  int nin = 0, ned = 0;
  for (int k = 0; k < n; ++k) {
    const int fin = edge_free_tiles(b.g[k].tiles_x, b.g[k].tiles_y) * 6 * b.slots[k];
    b.in0[k] = nin;
    b.ed0[k] = ned;
    nin += fin;
    ned += b.tm[k].total - fin;
  }
  b.in0[n] = nin;
  b.ed0[n] = ned;
  b.nin = nin;
  b.total = nin + ned;
}

int launch_stage(mcv_handle *h, int cand, int s, int c, bool pdl = true) {
  const StageLauncher &L = h->cands[cand];
  StageBatch<1> b;
  std::memset(&b, 0, sizeof(b));
  if (int rc = add_grid(b, 0, h, L, s, c)) return rc;
  number_items(b, 1);
  const int kind = stage_kind(h, s);
  const StageLaunchFn launch = h->active_ident ? L.launch_ident[kind] : L.launch[kind];
  if (!L.tma) {
    launch(dim3(b.g[0].tiles_x * b.g[0].tiles_y, 6, h->n_active), h->stream, b, pdl);
    return MCV_OK;
  }
  const int ctas = std::max(1, std::min(b.total, h->bps[cand] * h->nsm));
  launch(dim3(ctas), h->stream, b, pdl);
  return MCV_OK;
}

// Stage s of one RK step on every member: fused stage kernel, then the halo
// kernel on the stage's output.
int enqueue_stage(mcv_handle *h, int s, int c, cudaEvent_t mid = nullptr) {
  if (int rc = launch_stage(h, h->choice, s, c)) return rc;
  if (mid) cudaEventRecord(mid, h->stream);
  launch_halo(h, s, c);
  return MCV_OK;
}

// Time every candidate tile shape on this grid with the second stage kind,
// which does not modify its own inputs, and keep the fastest.
int autotune(mcv_handle *h) {
  if (h->choice >= 0) return MCV_OK;
  h->tune_ms.assign(h->ncands, -1.f);
  cudaEvent_t e0, e1;
  MCV_CUDA(cudaEventCreate(&e0), "event");
  MCV_CUDA(cudaEventCreate(&e1), "event");
  float best = 1e30f;
  int besti = 0;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < h->ncands && e == cudaSuccess; ++i) {
    // plain launches: each starts after the previous one has completed
    int rc = launch_stage(h, i, 1, h->cur, false);  // warm-up
    cudaEventRecord(e0, h->stream);
    for (int r = 0; r < 3 && !rc; ++r) rc = launch_stage(h, i, 1, h->cur, false);
    if (rc) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      return rc;
    }
    cudaEventRecord(e1, h->stream);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaGetLastError();
    h->tune_ms[i] = ms / 3.f;
    if (e == cudaSuccess && h->tune_ms[i] < best) {
      best = h->tune_ms[i];
      besti = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "autotune stage kernel");
  h->choice = besti;
  return MCV_OK;
}

int build_graphs(mcv_handle *h) {
  if (h->graph_exec[0]) return MCV_OK;
  if (int rc = autotune(h)) return rc;
  const int ngraphs = h->mixed ? 2 : 1;
  for (int c = 0; c < ngraphs; ++c) {
    MCV_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin step capture");
    int rc = MCV_OK;
    for (int s = 0; s < num_stages(h) && !rc; ++s) rc = enqueue_stage(h, s, c);
    cudaError_t le = cudaGetLastError();
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
    if (rc || le != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return rc ? rc : cuda_fail(le, "launch during step capture");
    }
    MCV_CUDA(ce, "end step capture");
    cudaError_t ie = cudaGraphInstantiate(&h->graph_exec[c], graph, 0);
    cudaGraphDestroy(graph);
    MCV_CUDA(ie, "instantiate step graph");
  }
  return MCV_OK;
}

// Checks the handle and lazily builds the step graphs.  With no active member
// a step enqueues nothing (*idle); callers that need a launch pass no flag.
int ready_to_step(mcv_handle *h, bool *idle = nullptr) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (!h->geometry_set) return fail(MCV_ERR_ORDER, "mcv_set_geometry must precede stepping");
  for (int k = 0; k < h->n_active; ++k)
    if (!h->member_set[h->active_host[k]])
      return fail(MCV_ERR_ORDER, "every active member must be set before stepping");
  if (h->n_active == 0) {
    if (!idle) return fail(MCV_ERR_ORDER, "no active member");
    *idle = true;
    return MCV_OK;
  }
  if (idle) *idle = false;
  return build_graphs(h);
}

// After nsteps of the active members: their step counts, and (split
// precision) the buffer now holding them.
void count_steps(mcv_handle *h, int nsteps) {
  for (int k = 0; k < h->n_active; ++k) {
    const int m = h->active_host[k];
    h->steps_done[m] += nsteps;
    if (h->mixed) h->mcur[m] = h->cur;
  }
}

// Enqueue nsteps replays of the step graph (split precision alternates the two).
int enqueue_steps(mcv_handle *h, int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    MCV_CUDA(cudaGraphLaunch(h->graph_exec[h->mixed ? h->cur : 0], h->stream), "launch step graph");
    if (h->mixed) h->cur = 1 - h->cur;
  }
  count_steps(h, nsteps);
  return MCV_OK;
}

// The state arrays of the current step.
// The state arrays holding member m.
double *const *state(mcv_handle *h, int m) { return h->mixed ? h->S[h->mcur[m]] : h->Y; }

}  // namespace

extern "C" const char *mcv_last_error(void) { return g_last_error.c_str(); }

extern "C" long long mcv_footprint_bytes(int order, int nc, int scheme, int precision, int members) {
  if ((order != 3 && order != 4) || nc < 2 || members < 1) return -1;
  if (precision != MCV_FP64 && precision != MCV_MIXED) return -1;
  GridDesc g{};
  int H, npx;
  grid_desc(order, nc, g, H, npx);
  return (long long)make_layout(g, H, scheme, precision, members).total;
}

extern "C" int mcv_device_memory(long long *free_bytes, long long *total_bytes) {
  if (!free_bytes || !total_bytes) return fail(MCV_ERR_ARG, "output is NULL");
  size_t f = 0, t = 0;
  MCV_CUDA(cudaMemGetInfo(&f, &t), "device memory");
  *free_bytes = (long long)f;
  *total_bytes = (long long)t;
  return MCV_OK;
}

extern "C" int mcv_create(int order, int nc, int scheme, int precision, double dt, double radius, int members,
                          mcv_handle **out) {
  if (!out) return fail(MCV_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (order != 3 && order != 4) return fail(MCV_ERR_ARG, "order must be 3 (MCV3) or 4 (MCV4)");
  if (nc < 2 || nc > 4096) return fail(MCV_ERR_ARG, "nc out of range [2, 4096]");
  if (scheme != MCV_RK3_TVD && scheme != MCV_RK4) return fail(MCV_ERR_ARG, "scheme must be MCV_RK3_TVD or MCV_RK4");
  if (precision != MCV_FP64 && precision != MCV_MIXED)
    return fail(MCV_ERR_ARG, "precision must be MCV_FP64 or MCV_MIXED");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(MCV_ERR_ARG, "dt must be positive and finite");
  if (!(radius > 0) || !std::isfinite(radius)) return fail(MCV_ERR_ARG, "radius must be positive and finite");
  if (members < 1) return fail(MCV_ERR_ARG, "members must be >= 1");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return fail(MCV_ERR_CUDA, "no CUDA device available (this library has no CPU path)");
  }
  int dev = 0;
  MCV_CUDA(cudaGetDevice(&dev), "get device");
  cudaDeviceProp prop;
  MCV_CUDA(cudaGetDeviceProperties(&prop, dev), "device properties");
  if (prop.major != 10) return fail(MCV_ERR_CUDA, "this library is built for sm_100a (B200) only");
  const int nsm = prop.multiProcessorCount;

  mcv_handle *h = new mcv_handle();
  h->order = order; h->nc = nc; h->scheme = scheme; h->precision = precision; h->members = members;
  h->mixed = precision == MCV_MIXED;
  h->dt = dt; h->radius = radius; h->device = dev;
  grid_desc(order, nc, h->g, h->H, h->npx);
  const double pi = 2.0 * std::asin(1.0);
  h->g.dx = (90. / nc) * (pi / 180.);
  h->g.inv_dx = 1. / h->g.dx;
  h->g.inv_2dx = 1. / (2. * h->g.dx);
  h->g.inv_dx2 = 1. / (h->g.dx * h->g.dx);
  h->dx2 = h->g.dx * h->g.dx;
  h->dx3 = std::pow(h->g.dx, 3.);
  h->member_set.assign(members, 0);
  h->steps_done.assign(members, 0);
  h->mcur.assign(members, 0);
  h->phibar_host.assign(members, 0.);
  h->cands = stage_launchers(order, h->mixed, &h->ncands);
  h->nsm = nsm;
  h->bps.assign(h->ncands, 0);
  for (int i = 0; i < h->ncands; ++i) {
    cudaError_t e = h->cands[i].prepare();
    if (e != cudaSuccess) {
      delete h;
      return cuda_fail(e, "set stage kernel shared memory");
    }
    h->bps[i] = h->cands[i].blocks_per_sm();
    if (h->bps[i] < 1) {
      delete h;
      return fail(MCV_ERR_CUDA, "a stage kernel candidate cannot be resident on an SM");
    }
  }
  int rc = upload_tables();
  if (rc) {
    delete h;
    return rc;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    return cuda_fail(e, "create stream");
  }
  const Layout L = make_layout(h->g, h->H, scheme, precision, members);
  e = cudaMalloc(&h->pool, L.total);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(h->stream);
    delete h;
    return fail(MCV_ERR_NOMEM, "device allocation failed (footprint exceeds free HBM)");
  }
  h->pool_bytes = L.total;
  char *base = (char *)h->pool;
  for (int k = 0; k < 3; ++k) {
    if (!h->mixed) {
      h->Y[k] = (double *)(base + L.f64_state[k]);
      h->A[k] = (double *)(base + L.f64_state[3 + k]);
      h->B[k] = (double *)(base + L.f64_state[6 + k]);
      h->acc[k] = scheme == MCV_RK4 ? (double *)(base + L.f64_acc[k]) : nullptr;
    } else {
      h->S[0][k] = (double *)(base + L.mix_state[k]);
      h->S[1][k] = (double *)(base + L.mix_state[3 + k]);
      h->DA[k] = (float *)(base + L.mix_inc[k]);
      h->DB[k] = (float *)(base + L.mix_inc[3 + k]);
      h->facc[k] = scheme == MCV_RK4 ? (float *)(base + L.mix_acc[k]) : nullptr;
    }
  }
  if (h->mixed) {
    h->phis32 = (float *)(base + L.phis32);
    h->bnd32 = (float4 *)(base + L.bnd32);
    h->met1d = (double4 *)(base + L.met1d);
    h->phibar = (double *)(base + L.phibar);
    h->prec = (double *)(base + L.prec);
  }
  h->sqrtG = (double *)(base + L.metric[0]);
  h->ig11 = (double *)(base + L.metric[1]);
  h->ig12 = (double *)(base + L.metric[2]);
  h->ig22 = (double *)(base + L.metric[3]);
  h->fcor = (double *)(base + L.metric[4]);
  h->phis = (double *)(base + L.phis);
  h->bnd = (double4 *)(base + L.bnd);
  h->Mtab = (double4 *)(base + L.M);
  h->Ntab = (double4 *)(base + L.N);
  h->giref = (int *)(base + L.iref);
  h->gcoef = (double2 *)(base + L.coef);
  h->partial = (double4 *)(base + L.partial);
  h->active = (int *)(base + L.active);
  h->flags = (int *)(base + L.flags);
  h->err = (int *)(base + L.err);
  h->stage = (double *)(base + L.stage);
  h->area = (double *)(base + L.area);
  // zero everything once: unused pitch padding and halo corners stay finite
  e = cudaMemsetAsync(h->pool, 0, L.total, h->stream);
  std::vector<double> area((size_t)nc * nc);
  equiangular_cell_areas(nc, radius, area.data());
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->area, area.data(), sizeof(double) * area.size(), cudaMemcpyHostToDevice, h->stream);
  // every member is active until mcv_set_active says otherwise
  h->active_host.resize(members);
  for (int m = 0; m < members; ++m) h->active_host[m] = m;
  h->n_active = members;
  h->active_ident = true;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h->active, h->active_host.data(), sizeof(int) * members, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    int r = cuda_fail(e, "clear device memory");
    mcv_destroy(h);
    return r;
  }
  *out = h;
  return MCV_OK;
}

extern "C" int mcv_destroy(mcv_handle *h) {
  if (!h) return MCV_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int c = 0; c < 2; ++c)
    if (h->graph_exec[c]) cudaGraphExecDestroy(h->graph_exec[c]);
  if (h->pool) cudaFree(h->pool);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MCV_OK;
}

extern "C" int mcv_set_geometry(mcv_handle *h, const double *sqrtG, const double *matrixG, const double *matrixIG,
                                const double *matrixA, const double *matrixIA, const double *f, const int *ghost_iref,
                                const double *ghost_coef) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (!sqrtG || !matrixG || !matrixIG || !matrixA || !matrixIA || !f || !ghost_iref || !ghost_coef)
    return fail(MCV_ERR_ARG, "geometry array is NULL");
  const int npx = h->npx, n = h->g.n, H = h->H, nc = h->nc;
  const size_t NP = (size_t)npx * npx * 6;
  std::vector<double> g11(NP), g12(NP), g22(NP);
  for (size_t k = 0; k < NP; ++k) {
    if (matrixIG[4 * k + 1] != matrixIG[4 * k + 2]) return fail(MCV_ERR_ARG, "matrixIG is not symmetric");
    g11[k] = matrixIG[4 * k + 0];
    g12[k] = matrixIG[4 * k + 2];  // IG(1,2) == IG(2,1) (projection_mod.F90:186)
    g22[k] = matrixIG[4 * k + 3];
  }
  // ghost weights: iref in 1..Nc, coef with coef**3. (ghost_mod.f90:222)
  std::vector<double2> coef((size_t)H * n);
  for (int hh = 0; hh < H; ++hh)
    for (int k = 0; k < n; ++k) {
      const int ir = ghost_iref[(size_t)hh * n + k];
      if (ir < 1 || ir > nc) return fail(MCV_ERR_ARG, "ghost_iref out of range 1..nc");
      const double c = ghost_coef[(size_t)hh * n + k];
      coef[(size_t)hh * n + k] = make_double2(c, std::pow(c, 3.));
    }
  // rotation matrices on the edge strips (convert_ghost_wind_P2SP / SP2P)
  std::vector<double4> Mt((size_t)24 * (H + 1) * n), Nt((size_t)24 * (H + 1) * n);
  for (int p = 0; p < 6; ++p)
    for (int e = 0; e < 4; ++e)
      for (int d = 0; d <= H; ++d)
        for (int k = 0; k < n; ++k) {
          auto pidx = [&](int dd) {
            int i, j;
            switch (e) {
              case 0: i = dd; j = k; break;
              case 1: i = n - 1 - dd; j = k; break;
              case 2: i = k; j = dd; break;
              default: i = k; j = n - 1 - dd; break;
            }
            return (size_t)(i + H) + (size_t)npx * ((size_t)(j + H) + (size_t)npx * p);
          };
          double m[4];
          const size_t in = pidx(d);
          matmul22(m, matrixA + 4 * in, matrixIG + 4 * in);
          Mt[((size_t)(p * 4 + e) * (H + 1) + d) * n + k] = make_double4(m[0], m[1], m[2], m[3]);
          const size_t out = pidx(-d);
          matmul22(m, matrixG + 4 * out, matrixIA + 4 * out);
          Nt[((size_t)(p * 4 + e) * (H + 1) + d) * n + k] = make_double4(m[0], m[1], m[2], m[3]);
        }
  std::vector<double4> met;
  if (h->mixed) {
    // 1-D metric table of the equiangular panel coordinate x_i = (i-1) dx/(D-1) + x_min
    // (mesh_mod.F90:135-136); the same table serves y because dx == dy.
    const double R = h->radius, D2R = (2.0 * std::asin(1.0)) / 180.;
    met.resize(npx);
    for (int i = 0; i < npx; ++i) {
      const double x = (double)(i + (1 - H) - 1) * h->g.dx / (double)(h->order - 1) + (-45. * D2R);
      const double t = std::tan(x), c = std::cos(x), s = std::sin(x);
      met[i] = make_double4(t, c * c / (R * R), s * c / R, R / (c * c));
    }
    // the kernels recompute sqrtG from this table: it must be the caller's
    // geometry (same radius), checked at the middle padded point of panel 1
    const int mid = npx / 2;
    const double4 mx = met[mid];
    const double rho2 = 1. + mx.x * mx.x + mx.x * mx.x;
    const double sg_table = mx.w * mx.w / (rho2 * std::sqrt(rho2));
    const size_t k = (size_t)mid + (size_t)npx * mid;
    if (std::fabs(sqrtG[k] / sg_table - 1.) > 1e-9)
      return fail(MCV_ERR_ARG, "radius does not match the geometry's sqrtG (mixed precision recomputes the metric)");
  }
  int rc;
  if ((rc = upload_padded(h, h->sqrtG, sqrtG, 8))) return rc;
  if ((rc = upload_padded(h, h->ig11, g11.data(), 8))) return rc;
  if ((rc = upload_padded(h, h->ig12, g12.data(), 8))) return rc;
  if ((rc = upload_padded(h, h->ig22, g22.data(), 8))) return rc;
  if ((rc = upload_padded(h, h->fcor, f, 8))) return rc;
  MCV_CUDA(cudaMemcpyAsync(h->Mtab, Mt.data(), Mt.size() * sizeof(double4), cudaMemcpyHostToDevice, h->stream),
           "upload Mtab");
  MCV_CUDA(cudaMemcpyAsync(h->Ntab, Nt.data(), Nt.size() * sizeof(double4), cudaMemcpyHostToDevice, h->stream),
           "upload Ntab");
  MCV_CUDA(cudaMemcpyAsync(h->giref, ghost_iref, sizeof(int) * (size_t)H * n, cudaMemcpyHostToDevice, h->stream),
           "upload iref");
  MCV_CUDA(cudaMemcpyAsync(h->gcoef, coef.data(), sizeof(double2) * coef.size(), cudaMemcpyHostToDevice, h->stream),
           "upload coef");
  if (h->mixed)
    MCV_CUDA(cudaMemcpyAsync(h->met1d, met.data(), sizeof(double4) * npx, cudaMemcpyHostToDevice, h->stream),
             "upload metric table");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "geometry upload");
  h->sqrtG_host.assign(sqrtG, sqrtG + NP);
  h->geometry_set = true;
  return MCV_OK;
}

extern "C" int mcv_set_geometry_equiangular(mcv_handle *h) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (!(h->radius > 0.)) return fail(MCV_ERR_ARG, "the handle's radius must be positive");
  const double pi = 2.0 * std::asin(1.0);
  GeomArgs a{};
  a.order = h->order;
  a.nc = h->nc;
  a.npx = h->npx;
  a.n = h->g.n;
  a.H = h->H;
  a.P = h->g.P;
  a.radius = h->radius;
  a.dx = h->g.dx;  // (90 / nc) degrees in radians, as the host builder
  a.x_min = -45. * (pi / 180.);
  a.pi = pi;
  a.sqrtG = h->sqrtG;
  a.ig11 = h->ig11;
  a.ig12 = h->ig12;
  a.ig22 = h->ig22;
  a.fcor = h->fcor;
  a.Mtab = h->Mtab;
  a.Ntab = h->Ntab;
  a.giref = h->giref;
  a.gcoef = h->gcoef;
  a.met1d = h->mixed ? h->met1d : nullptr;
  a.err = h->err;
  MCV_CUDA(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream), "clear error flag");
  if (int e = build_geometry_device(a, h->stream))
    return fail(MCV_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
  int bad = 0;
  MCV_CUDA(cudaMemcpyAsync(&bad, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "read error flag");
  MCV_CUDA(cudaMemsetAsync(h->err, 0, sizeof(int), h->stream), "clear error flag");
  const size_t NP = (size_t)h->npx * h->npx * 6;
  h->sqrtG_host.resize(NP);
  if (int rc = download_padded(h, h->sqrtG_host.data(), h->sqrtG)) return rc;
  MCV_CUDA(cudaStreamSynchronize(h->stream), "device geometry");
  if (bad) return fail(MCV_ERR_ARG, "ghost cell location error");
  h->geometry_set = true;
  return MCV_OK;
}

extern "C" int mcv_get_geometry(mcv_handle *h, double *sqrtG, double *ig11, double *ig12, double *ig22, double *f,
                                int *ghost_iref, double *ghost_coef) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (!h->geometry_set) return fail(MCV_ERR_ORDER, "no geometry set");
  int rc;
  const double *src[5] = {h->sqrtG, h->ig11, h->ig12, h->ig22, h->fcor};
  double *dst[5] = {sqrtG, ig11, ig12, ig22, f};
  for (int k = 0; k < 5; ++k)
    if (dst[k] && (rc = download_padded(h, dst[k], src[k]))) return rc;
  const size_t nh = (size_t)h->H * h->g.n;
  std::vector<double2> coef(ghost_coef ? nh : 0);
  if (ghost_iref)
    MCV_CUDA(cudaMemcpyAsync(ghost_iref, h->giref, sizeof(int) * nh, cudaMemcpyDeviceToHost, h->stream),
             "download iref");
  if (ghost_coef)
    MCV_CUDA(cudaMemcpyAsync(coef.data(), h->gcoef, sizeof(double2) * nh, cudaMemcpyDeviceToHost, h->stream),
             "download coef");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "download geometry");
  for (size_t k = 0; k < coef.size(); ++k) ghost_coef[k] = coef[k].x;
  return MCV_OK;
}

extern "C" int mcv_set_member(mcv_handle *h, int m, const double *phi_s, const double *u, const double *v,
                              const double *phi) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (!phi_s || !u || !v || !phi) return fail(MCV_ERR_ARG, "state array is NULL");
  if (!h->geometry_set) return fail(MCV_ERR_ORDER, "mcv_set_geometry must precede mcv_set_member");
  const long long off = (long long)m * h->g.mstride;
  if (h->mixed) h->mcur[m] = h->cur;
  double *const *Y = state(h, m);
  int rc;
  if ((rc = upload_padded(h, h->phis + off, phi_s, 8))) return rc;
  if ((rc = upload_padded(h, Y[0] + off, u, 8))) return rc;
  if ((rc = upload_padded(h, Y[1] + off, v, 8))) return rc;
  if ((rc = upload_padded(h, Y[2] + off, phi, 8))) return rc;
  std::vector<float> ps;
  if (h->mixed) {
    const int npx = h->npx, H = h->H, n = h->g.n;
    const size_t NP = (size_t)npx * npx * 6;
    ps.resize(NP);
    for (size_t k = 0; k < NP; ++k) ps[k] = (float)phi_s[k];
    // mean depth: sqrtG-weighted mean of phi over the interior points
    double num = 0., den = 0.;
    for (int p = 0; p < 6; ++p)
      for (int j = H; j < H + n; ++j)
        for (int i = H; i < H + n; ++i) {
          const size_t k = (size_t)i + (size_t)npx * ((size_t)j + (size_t)npx * p);
          num += h->sqrtG_host[k] * phi[k];
          den += h->sqrtG_host[k];
        }
    h->phibar_host[m] = num / den;
    if ((rc = upload_padded(h, h->phis32 + off, ps.data(), 4))) return rc;
    MCV_CUDA(cudaMemcpyAsync(h->phibar + m, &h->phibar_host[m], sizeof(double), cudaMemcpyHostToDevice, h->stream),
             "upload mean depth");
  }
  MCV_CUDA(cudaStreamSynchronize(h->stream), "member upload");
  h->member_set[m] = 1;
  h->steps_done[m] = 0;
  return MCV_OK;
}

namespace {

// Compensated total of the per-block partial sums {s1, c1, s2, c2} (fixed
// order: the same bits on every call).
int sum_partials(mcv_handle *h, double &s1, double &s2) {
  std::vector<double4> part(kPartialBlocks);
  MCV_CUDA(cudaMemcpyAsync(part.data(), h->partial, sizeof(double4) * kPartialBlocks, cudaMemcpyDeviceToHost,
                           h->stream),
           "download partial sums");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "partial sums");
  KSum a{0., 0.}, b{0., 0.};
  auto add = [](KSum &k, double x) {
    const double t = k.s + x;
    if (std::fabs(k.s) >= std::fabs(x)) k.c += (k.s - t) + x;
    else k.c += (x - t) + k.s;
    k.s = t;
  };
  for (const double4 &q : part) {
    add(a, q.x);
    a.c += q.y;
    add(b, q.z);
    b.c += q.w;
  }
  s1 = a.s + a.c;
  s2 = b.s + b.c;
  return MCV_OK;
}

}  // namespace

extern "C" int mcv_set_member_balanced_flow(mcv_handle *h, int m, double gh0, double u0, double alpha, int lmax,
                                            const double *coef, double rms, double mountain_h0, double lon_c,
                                            double lat_c, double efold) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (!h->geometry_set) return fail(MCV_ERR_ORDER, "the geometry must precede the member's initial state");
  if (lmax < 0 || lmax > 200 || (lmax > 0 && !coef)) return fail(MCV_ERR_ARG, "bad harmonic arguments");
  if (mountain_h0 > 0. && !(efold > 0.)) return fail(MCV_ERR_ARG, "bad mountain arguments");
  const long long off = (long long)m * h->g.mstride;
  if (h->mixed) h->mcur[m] = h->cur;
  double *const *Y = state(h, m);
  const double pi = 2.0 * std::asin(1.0);
  IcArgs a{};
  a.order = h->order;
  a.nc = h->nc;
  a.npx = h->npx;
  a.n = h->g.n;
  a.H = h->H;
  a.P = h->g.P;
  a.radius = h->radius;
  a.dx = h->g.dx;
  a.x_min = -45. * (pi / 180.);
  a.pi = pi;
  a.gh0 = gh0;
  a.u0 = u0;
  a.alpha = alpha;
  a.mountain = mountain_h0 > 0.;
  a.h0 = mountain_h0;
  a.lon_c = lon_c;
  a.lat_c = lat_c;
  a.efold = efold;
  a.u = Y[0] + off;
  a.v = Y[1] + off;
  a.phi = Y[2] + off;
  a.phis = h->phis + off;
  a.phis32 = h->mixed ? h->phis32 + off : nullptr;
  a.sqrtG = h->sqrtG;
  double *dcoef = nullptr;
  int rc;
  if (lmax > 0 && rms != 0.) {
    const size_t nb = sizeof(double) * (size_t)(lmax + 1) * (lmax + 1);
    MCV_CUDA(cudaMallocAsync((void **)&dcoef, nb, h->stream), "coefficients");
    MCV_CUDA(cudaMemcpyAsync(dcoef, coef, nb, cudaMemcpyHostToDevice, h->stream), "upload coefficients");
    a.coef = dcoef;
    a.lmax = lmax;
    // unit-scale height, then its area-weighted RMS (cases.harmonic_height)
    int e = ic_harmonics_device(a, h->stream);
    if (!e) e = ic_sums_device(a, 0, a.phis, h->partial, kPartialBlocks, h->stream);
    if (e) {
      cudaFreeAsync(dcoef, h->stream);
      return fail(MCV_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    }
    double swh2 = 0., sw = 0.;
    if ((rc = sum_partials(h, swh2, sw))) return rc;
    const double area_rms = std::sqrt(swh2 / sw);
    if (!(area_rms > 0.)) {
      cudaFreeAsync(dcoef, h->stream);
      return fail(MCV_ERR_ARG, "the harmonic coefficients give a zero field");
    }
    a.ratio = rms / area_rms;
  }
  int e = ic_fields_device(a, h->stream);
  if (dcoef) cudaFreeAsync(dcoef, h->stream);
  if (e) return fail(MCV_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
  if (h->mixed) {
    // mean depth: sqrtG-weighted mean of phi over the interior points
    if ((e = ic_sums_device(a, 1, a.phi, h->partial, kPartialBlocks, h->stream)))
      return fail(MCV_ERR_CUDA, cudaGetErrorString((cudaError_t)e));
    double num = 0., den = 0.;
    if ((rc = sum_partials(h, num, den))) return rc;
    h->phibar_host[m] = num / den;
    MCV_CUDA(cudaMemcpyAsync(h->phibar + m, &h->phibar_host[m], sizeof(double), cudaMemcpyHostToDevice, h->stream),
             "upload mean depth");
  }
  MCV_CUDA(cudaStreamSynchronize(h->stream), "member initial state");
  h->member_set[m] = 1;
  h->steps_done[m] = 0;
  return MCV_OK;
}

extern "C" int mcv_set_state(mcv_handle *h, int m, const double *u, const double *v, const double *phi) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (!u || !v || !phi) return fail(MCV_ERR_ARG, "state array is NULL");
  if (!h->member_set[m]) return fail(MCV_ERR_ORDER, "mcv_set_member must precede mcv_set_state");
  const long long off = (long long)m * h->g.mstride;
  if (h->mixed) h->mcur[m] = h->cur;
  double *const *Y = state(h, m);
  int rc;
  if ((rc = upload_padded(h, Y[0] + off, u, 8))) return rc;
  if ((rc = upload_padded(h, Y[1] + off, v, 8))) return rc;
  if ((rc = upload_padded(h, Y[2] + off, phi, 8))) return rc;
  MCV_CUDA(cudaStreamSynchronize(h->stream), "state upload");
  h->steps_done[m] = 0;
  return MCV_OK;
}

extern "C" int mcv_step_async(mcv_handle *h, int nsteps) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (nsteps < 0) return fail(MCV_ERR_ARG, "nsteps must be >= 0");
  bool idle = false;
  if (int rc = ready_to_step(h, &idle)) return rc;
  if (idle) return MCV_OK;
  return enqueue_steps(h, nsteps);
}

extern "C" int mcv_sync(mcv_handle *h) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "step");
  int err = 0;
  MCV_CUDA(cudaMemcpy(&err, h->err, sizeof(int), cudaMemcpyDeviceToHost), "read stage error flag");
  if (err) return fail(MCV_ERR_CUDA, "stage kernel: a staged tile's copies did not arrive in time");
  return MCV_OK;
}

namespace {

// Failure path of the stage kernels' bounded copy wait (mbar_wait_bounded),
// run without a GPU fault: one warp waits on a fresh mbarrier; with `complete`
// thread 0 arrives first and the wait must succeed at once, otherwise nothing
// ever arrives and the wait must give up after limit_ns and say so, as the
// stage kernel does before it raises its error flag and returns.
__global__ void wait_selftest_kernel(int complete, unsigned long long limit_ns, int *timed_out,
                                     unsigned long long *elapsed_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (complete && threadIdx.x == 0) mbar_arrive(&bar);
  __syncthreads();  // the arrival, if any, precedes every wait
  const uint64_t t0 = global_ns();
  const bool got = mbar_wait_bounded(&bar, 0u, limit_ns);
  const uint64_t t1 = global_ns();
  if (__syncthreads_or(!got) && threadIdx.x == 0) *timed_out = 1;
  if (threadIdx.x == 0) *elapsed_ns = t1 - t0;
}

}  // namespace

extern "C" int mcv_selftest_wait(int complete, double limit_ms, int *timed_out, double *elapsed_ms) {
  if (!timed_out || !elapsed_ms) return fail(MCV_ERR_ARG, "output pointer is NULL");
  if (!(limit_ms > 0.) || limit_ms > 2000.) return fail(MCV_ERR_ARG, "limit_ms must be in (0, 2000]");
  struct Out {
    int timed_out;
    int pad;
    unsigned long long elapsed_ns;
  };
  Out *d = nullptr;
  MCV_CUDA(cudaMalloc((void **)&d, sizeof(Out)), "self-test buffer");
  Out o{};
  cudaError_t e = cudaMemset(d, 0, sizeof(Out));
  if (e == cudaSuccess) {
    wait_selftest_kernel<<<1, 32>>>(complete, (unsigned long long)(limit_ms * 1e6), &d->timed_out, &d->elapsed_ns);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&o, d, sizeof(Out), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "wait self-test");
  *timed_out = o.timed_out;
  *elapsed_ms = (double)o.elapsed_ns * 1e-6;
  return MCV_OK;
}

extern "C" int mcv_query(mcv_handle *h) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  const cudaError_t e = cudaStreamQuery(h->stream);
  if (e == cudaSuccess) return MCV_OK;
  if (e == cudaErrorNotReady) {
    cudaGetLastError();
    return MCV_BUSY;
  }
  return cuda_fail(e, "query");
}

extern "C" int mcv_check_finite(mcv_handle *h, int *flags) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  MCV_CUDA(cudaMemsetAsync(h->flags, 0, sizeof(int) * h->members, h->stream), "clear flags");
  for (int m = 0; m < h->members; ++m) {
    // one launch per member: split-precision members may sit in different buffers
    double *const *y = state(h, m);
    const long long off = (long long)m * h->g.mstride;
    finite_check_kernel<<<148, 256, 0, h->stream>>>(h->g, h->H, y[0] + off, y[1] + off, y[2] + off, h->flags + m);
  }
  MCV_CUDA(cudaGetLastError(), "launch finite check");
  std::vector<int> f(h->members);
  MCV_CUDA(cudaMemcpyAsync(f.data(), h->flags, sizeof(int) * h->members, cudaMemcpyDeviceToHost, h->stream),
           "download flags");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "finite check");
  if (flags)
    for (int m = 0; m < h->members; ++m) flags[m] = f[m];
  for (int k = 0; k < h->n_active; ++k)
    if (f[h->active_host[k]]) return fail(MCV_ERR_NONFINITE, "an active member's state is not finite");
  return MCV_OK;
}

extern "C" int mcv_set_active(mcv_handle *h, int count, const int *members) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (count < 0 || count > h->members) return fail(MCV_ERR_ARG, "active count out of range [0, members]");
  if (count > 0 && !members) return fail(MCV_ERR_ARG, "members is NULL");
  std::vector<char> seen(h->members, 0);
  for (int k = 0; k < count; ++k) {
    const int m = members[k];
    if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "active member index out of range");
    if (seen[m]) return fail(MCV_ERR_ARG, "active member listed twice");
    seen[m] = 1;
  }
  bool ident = true;
  for (int k = 0; k < count; ++k) ident = ident && members[k] == k;
  if (count != h->n_active || ident != h->active_ident) {
    // the step graphs hold the launch grids and whether the list is the
    // identity: rebuild before the next step
    MCV_CUDA(cudaStreamSynchronize(h->stream), "drain before changing the active set");
    for (int c = 0; c < 2; ++c)
      if (h->graph_exec[c]) {
        cudaGraphExecDestroy(h->graph_exec[c]);
        h->graph_exec[c] = nullptr;
      }
  }
  for (int k = 0; k < count; ++k) {
    const int m = members[k];
    h->active_host[k] = m;
    if (h->mixed && h->mcur[m] != h->cur) {
      // a member left out of earlier steps sits in the other buffer: move it
      // to the one the next step reads
      const size_t bytes = (size_t)h->g.mstride * sizeof(double);
      const long long off = (long long)m * h->g.mstride;
      for (int f = 0; f < 3; ++f)
        MCV_CUDA(cudaMemcpyAsync(h->S[h->cur][f] + off, h->S[h->mcur[m]][f] + off, bytes, cudaMemcpyDeviceToDevice,
                                 h->stream),
                 "move member state");
      h->mcur[m] = h->cur;
    }
  }
  h->n_active = count;
  h->active_ident = ident;
  // ordered after the steps already enqueued on the handle's stream; a copy
  // from pageable memory has consumed the host list when it returns
  if (count > 0)
    MCV_CUDA(cudaMemcpyAsync(h->active, h->active_host.data(), sizeof(int) * count, cudaMemcpyHostToDevice,
                             h->stream),
             "upload active members");
  return MCV_OK;
}

extern "C" int mcv_step(mcv_handle *h, int nsteps) {
  if (int rc = mcv_step_async(h, nsteps)) return rc;
  return mcv_sync(h);
}

extern "C" int mcv_get_state(mcv_handle *h, int m, double *u, double *v, double *phi, double *phiG) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  const long long off = (long long)m * h->g.mstride;
  const size_t NP = (size_t)h->npx * h->npx * 6;
  std::vector<double> tmp;
  double *phi_dst = phi;
  if (!phi && phiG) {
    tmp.resize(NP);
    phi_dst = tmp.data();
  }
  double *const *Y = state(h, m);
  int rc;
  if (u && (rc = download_padded(h, u, Y[0] + off))) return rc;
  if (v && (rc = download_padded(h, v, Y[1] + off))) return rc;
  if (phi_dst && (rc = download_padded(h, phi_dst, Y[2] + off))) return rc;
  MCV_CUDA(cudaStreamSynchronize(h->stream), "state download");
  if (h->steps_done[m] > 0) {
    // Halo corners are never computed: phi holds FillValue there after
    // correct_bdy_ghost (ghost_mod.f90:161,179) and the history output marks
    // u and v the same way (addFillValue, output_mod.F90:230-248).
    const int npx = h->npx, H = h->H;
    double *fields[3] = {u, v, phi_dst};
    for (double *fld : fields) {
      if (!fld) continue;
      for (int p = 0; p < 6; ++p)
        for (int cj = 0; cj < 2; ++cj)  // the four H x H corner squares of each panel
          for (int ci = 0; ci < 2; ++ci)
            for (int j = 0; j < H; ++j)
              for (int i = 0; i < H; ++i) {
                const size_t ii = ci ? (size_t)(npx - H + i) : (size_t)i, jj = cj ? (size_t)(npx - H + j) : (size_t)j;
                fld[ii + (size_t)npx * (jj + (size_t)npx * p)] = -9999999999999999.;
              }
    }
  }
  if (phiG)
    for (size_t k = 0; k < NP; ++k) phiG[k] = phi_dst[k] * h->sqrtG_host[k];
  return MCV_OK;
}

extern "C" int mcv_mass_energy(mcv_handle *h, int m, double *mass, double *energy) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (!h->geometry_set || !h->member_set[m]) return fail(MCV_ERR_ORDER, "geometry and member must be set");
  const long long off = (long long)m * h->g.mstride;
  const double w0 = 1., w1 = (h->order == 3) ? 4. : 3., wden = (h->order == 3) ? 36. : 80.;
  double *const *Y = state(h, m);
  if (h->order == 3)
    mass_energy_kernel<3><<<kPartialBlocks, 256, 0, h->stream>>>(h->g, Y[0] + off, Y[1] + off, Y[2] + off, h->sqrtG,
                                                                 h->ig11, h->ig12, h->ig22, h->phis + off, w0, w1,
                                                                 wden, h->partial);
  else
    mass_energy_kernel<4><<<kPartialBlocks, 256, 0, h->stream>>>(h->g, Y[0] + off, Y[1] + off, Y[2] + off, h->sqrtG,
                                                                 h->ig11, h->ig12, h->ig22, h->phis + off, w0, w1,
                                                                 wden, h->partial);
  MCV_CUDA(cudaGetLastError(), "launch mass/energy");
  std::vector<double4> part(kPartialBlocks);
  MCV_CUDA(cudaMemcpyAsync(part.data(), h->partial, sizeof(double4) * kPartialBlocks, cudaMemcpyDeviceToHost,
                           h->stream),
           "download partial sums");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "mass/energy");
  KSum ms{0., 0.}, es{0., 0.};
  auto add = [](KSum &a, double x) {
    const double t = a.s + x;
    if (std::fabs(a.s) >= std::fabs(x)) a.c += (a.s - t) + x;
    else a.c += (x - t) + a.s;
    a.s = t;
  };
  for (const double4 &q : part) {
    add(ms, q.x);
    ms.c += q.y;
    add(es, q.z);
    es.c += q.w;
  }
  if (mass) *mass = ms.s + ms.c;
  if (energy) *energy = es.s + es.c;
  return MCV_OK;
}

namespace {

// The equiangular sqrtG of the handle's radius at the middle padded point of
// panel 1 agrees with the geometry the handle holds (device formulas that
// take the radius -- the history's A IG -- need the caller's radius).
bool radius_matches(const mcv_handle *h) {
  const int npx = h->npx, mid = npx / 2;
  const double pi = 2.0 * std::asin(1.0);
  const double x = (double)(mid + (1 - h->H) - 1) * h->g.dx / (double)(h->order - 1) + (-45. * pi / 180.);
  const double t = std::tan(x), c = std::cos(x);
  const double rho2 = 1. + 2. * t * t;
  const double sg = h->radius * h->radius / (c * c * c * c * rho2 * std::sqrt(rho2));
  const size_t k = (size_t)mid + (size_t)npx * mid;
  return k < h->sqrtG_host.size() && std::fabs(h->sqrtG_host[k] / sg - 1.) <= 1e-9;
}

GeomArgs history_args(const mcv_handle *h) {
  GeomArgs a{};
  a.order = h->order;
  a.nc = h->nc;
  a.npx = h->npx;
  a.n = h->g.n;
  a.H = h->H;
  a.P = h->g.P;
  a.radius = h->radius;
  a.dx = h->g.dx;
  a.pi = 2.0 * std::asin(1.0);
  a.x_min = -45. * (a.pi / 180.);
  return a;
}

// FillValue (src/constants_mod.F90:20) in the four H x H halo corner squares
// of a padded host field of the handle's grid.
void fill_corners(const mcv_handle *h, double *fld) {
  const int npx = h->npx, H = h->H;
  for (int p = 0; p < 6; ++p)
    for (int cj = 0; cj < 2; ++cj)
      for (int ci = 0; ci < 2; ++ci)
        for (int j = 0; j < H; ++j)
          for (int i = 0; i < H; ++i) {
            const size_t ii = ci ? (size_t)(npx - H + i) : (size_t)i, jj = cj ? (size_t)(npx - H + j) : (size_t)j;
            fld[ii + (size_t)npx * (jj + (size_t)npx * p)] = -9999999999999999.;
          }
}

}  // namespace

extern "C" int mcv_get_history(mcv_handle *h, int m, double *u, double *v, double *phi, double *zonal, double *merid,
                               double *uC, double *vC, double *phiC) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (!h->geometry_set || !h->member_set[m]) return fail(MCV_ERR_ORDER, "geometry and member must be set");
  if ((zonal || merid) && !radius_matches(h))
    return fail(MCV_ERR_ARG, "the handle's radius does not match its geometry (the wind rotation needs it)");
  const long long off = (long long)m * h->g.mstride;
  double *const *Y = state(h, m);
  const size_t field = (size_t)h->npx * h->npx * 6 * sizeof(double);
  int rc;
  if (u && (rc = download_padded(h, u, Y[0] + off))) return rc;
  if (v && (rc = download_padded(h, v, Y[1] + off))) return rc;
  if (phi && (rc = download_padded(h, phi, Y[2] + off))) return rc;
  const GeomArgs ga = history_args(h);
  double *const wind[2] = {zonal, merid};
  for (int which = 0; which < 2; ++which) {
    if (!wind[which]) continue;
    // the staging field is free again once the previous copy out has run
    if (int e = history_p2sp_device(ga, Y[0] + off, Y[1] + off, which, h->stage, h->stream))
      return cuda_fail((cudaError_t)e, "history wind rotation");
    MCV_CUDA(cudaMemcpyAsync(wind[which], h->stage, field, cudaMemcpyDeviceToHost, h->stream), "download wind");
  }
  double *const cells[3] = {uC, vC, phiC};
  const size_t ncell = (size_t)(h->nc + 2) * (h->nc + 2) * 6;
  for (int f = 0; f < 3; ++f) {
    if (!cells[f]) continue;
    if (int e = via_device(h->order, h->nc, h->npx, h->g.P, Y[f] + off, h->stage, h->stream))
      return cuda_fail((cudaError_t)e, "cell averages");
    MCV_CUDA(cudaMemcpyAsync(cells[f], h->stage, ncell * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
             "download cell averages");
  }
  MCV_CUDA(cudaStreamSynchronize(h->stream), "history download");
  // addFillValue (output_mod.F90:230-248) on u, v; phi's corners hold FillValue
  // once a step's correct_bdy_ghost has run (ghost_mod.f90:161,179)
  if (u) fill_corners(h, u);
  if (v) fill_corners(h, v);
  if (phi && h->steps_done[m] > 0) fill_corners(h, phi);
  return MCV_OK;
}

extern "C" int mcv_height_error_norms(mcv_handle *a, int ma, mcv_handle *b, int mb, double *norms) {
  if (!a || !b || !norms) return fail(MCV_ERR_ARG, "handle or output is NULL");
  if (ma < 0 || ma >= a->members || mb < 0 || mb >= b->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (a->order != b->order || a->nc != b->nc) return fail(MCV_ERR_ARG, "the two handles hold different grids");
  if (a->device != b->device) return fail(MCV_ERR_ARG, "the two handles live on different devices");
  if (!a->member_set[ma] || !b->member_set[mb]) return fail(MCV_ERR_ORDER, "both members must be set");
  // b's queued steps come first
  if (a != b) MCV_CUDA(cudaStreamSynchronize(b->stream), "wait for the reference handle");
  const double *pa = state(a, ma)[2] + (long long)ma * a->g.mstride;
  const double *pb = state(b, mb)[2] + (long long)mb * b->g.mstride;
  const int blocks = kPartialBlocks / 2;
  if (int e = norms_device(a->order, a->nc, a->npx, a->g.P, pa, pb, a->area, a->partial, blocks, a->stream))
    return cuda_fail((cudaError_t)e, "error norms");
  std::vector<double4> part(kPartialBlocks);
  MCV_CUDA(cudaMemcpyAsync(part.data(), a->partial, sizeof(double4) * kPartialBlocks, cudaMemcpyDeviceToHost,
                           a->stream),
           "download norm partials");
  MCV_CUDA(cudaStreamSynchronize(a->stream), "error norms");
  double l1 = 0., r1 = 0., l2 = 0., r2 = 0., md = 0., mbx = 0.;
  for (int k = 0; k < blocks; ++k) {
    l1 += part[2 * k].x;
    r1 += part[2 * k].y;
    l2 += part[2 * k].z;
    r2 += part[2 * k].w;
    md = std::max(md, part[2 * k + 1].x);
    mbx = std::max(mbx, part[2 * k + 1].y);
  }
  norms[0] = l1 / r1;
  norms[1] = std::sqrt(l2 / r2);
  norms[2] = md / mbx;
  return MCV_OK;
}

extern "C" int mcv_cell_areas(int nc, double radius, double *areaCell) {
  if (nc < 2 || nc > 4096 || !(radius > 0.) || !areaCell) return fail(MCV_ERR_ARG, "bad cell-area arguments");
  std::vector<double> a((size_t)nc * nc);
  equiangular_cell_areas(nc, radius, a.data());
  const int nce = nc + 2;
  for (int p = 0; p < 6; ++p)
    for (int j = 0; j < nce; ++j)
      for (int i = 0; i < nce; ++i) {
        const bool in = i >= 1 && i <= nc && j >= 1 && j <= nc;
        areaCell[(size_t)i + (size_t)nce * ((size_t)j + (size_t)nce * p)] =
            in ? a[(size_t)(i - 1) + (size_t)nc * (j - 1)] : 0.;
      }
  return MCV_OK;
}

extern "C" int mcv_time_steps(mcv_handle *h, int nsteps, double *ms) {
  if (int rc = ready_to_step(h)) return rc;
  if (nsteps < 1 || !ms) return fail(MCV_ERR_ARG, "nsteps >= 1 and ms required");
  cudaEvent_t e0, e1;
  MCV_CUDA(cudaEventCreate(&e0), "event");
  MCV_CUDA(cudaEventCreate(&e1), "event");
  cudaEventRecord(e0, h->stream);
  int rc = enqueue_steps(h, nsteps);
  cudaEventRecord(e1, h->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "timed steps");
  *ms = t;
  return MCV_OK;
}

extern "C" int mcv_profile_step(mcv_handle *h, int nsteps, double *stage_ms, double *halo_ms) {
  if (int rc = ready_to_step(h)) return rc;
  if (nsteps < 1 || !stage_ms || !halo_ms) return fail(MCV_ERR_ARG, "nsteps >= 1 and outputs required");
  const int S = num_stages(h);
  std::vector<cudaEvent_t> ev((size_t)nsteps * S * 3);
  for (auto &e : ev) MCV_CUDA(cudaEventCreate(&e), "event");
  for (int it = 0; it < nsteps; ++it) {
    for (int s = 0; s < S; ++s) {
      cudaEvent_t *e = &ev[((size_t)it * S + s) * 3];
      cudaEventRecord(e[0], h->stream);
      if (int rc = enqueue_stage(h, s, h->cur, e[1])) {
        cudaStreamSynchronize(h->stream);
        for (auto &ev_ : ev) cudaEventDestroy(ev_);
        return rc;
      }
      cudaEventRecord(e[2], h->stream);
    }
    if (h->mixed) h->cur = 1 - h->cur;
  }
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
  double st[4] = {0, 0, 0, 0}, ha = 0;
  for (int it = 0; it < nsteps && err == cudaSuccess; ++it)
    for (int s = 0; s < S; ++s) {
      cudaEvent_t *e = &ev[((size_t)it * S + s) * 3];
      float a = 0, b = 0;
      cudaEventElapsedTime(&a, e[0], e[1]);
      cudaEventElapsedTime(&b, e[1], e[2]);
      st[s] += a;
      ha += b;
    }
  for (auto &e : ev) cudaEventDestroy(e);
  if (err != cudaSuccess) return cuda_fail(err, "profiled steps");
  for (int s = 0; s < 4; ++s) stage_ms[s] = s < S ? st[s] / nsteps : 0.;
  *halo_ms = ha / ((double)nsteps * S);
  count_steps(h, nsteps);
  return MCV_OK;
}

extern "C" int mcv_tuning(mcv_handle *h, int *ncand, int *chosen, int *shapes, float *ms) {
  if (int rc = ready_to_step(h)) return rc;
  if (ncand) *ncand = h->ncands;
  if (chosen) *chosen = h->choice;
  for (int i = 0; i < h->ncands; ++i) {
    if (shapes) {
      shapes[6 * i] = h->cands[i].CX;
      shapes[6 * i + 1] = h->cands[i].CY;
      shapes[6 * i + 2] = h->cands[i].NT;
      shapes[6 * i + 3] = h->cands[i].walk;
      shapes[6 * i + 4] = h->cands[i].minb;
      shapes[6 * i + 5] = h->cands[i].tma ? 1 : 0;
    }
    if (ms) ms[i] = h->tune_ms[i];
  }
  return MCV_OK;
}

extern "C" int mcv_select_tile(mcv_handle *h, int index) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (index < -1 || index >= h->ncands) return fail(MCV_ERR_ARG, "tile index out of range");
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (int c = 0; c < 2; ++c)
    if (h->graph_exec[c]) {
      cudaGraphExecDestroy(h->graph_exec[c]);
      h->graph_exec[c] = nullptr;
    }
  h->choice = index;  // -1: autotune again before the next step
  if (index >= 0 && (int)h->tune_ms.size() != h->ncands) h->tune_ms.assign(h->ncands, -1.f);
  return MCV_OK;
}

// ---------------------------------------------------------------------------
// Groups: several handles (grids of one order, arithmetic and scheme, any Nc,
// dt and members) advanced together, each stage one batched launch of the
// stage kernel over all of them followed by each grid's halo kernel.
// ---------------------------------------------------------------------------
struct mcv_group {
  std::vector<mcv_handle *> hs;
  int cand = -1;  // stage-kernel candidate every grid of the group uses
  int bps = 0;    // resident CTAs per SM of the batched kernel
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> ready;  // per handle: work queued on its own stream before a group step
  // step graphs: built for the members' buffer parities `key_cur` (and their
  // complement, which the next step has), active counts `key_active` and
  // whether each active list is the identity `key_ident`
  cudaGraphExec_t graph[2]{};
  std::vector<mcv_handle *> key_hs;  // the handles with active members the graphs advance
  std::vector<int> key_cur, key_active, key_ident;
};

namespace {

void drop_group_graphs(mcv_group *g) {
  if (g->graph[0] || g->graph[1]) cudaStreamSynchronize(g->stream);  // launches still queued end first
  for (int c = 0; c < 2; ++c)
    if (g->graph[c]) {
      cudaGraphExecDestroy(g->graph[c]);
      g->graph[c] = nullptr;
    }
}

// One stage of the group's step (handles with active members only), with each
// handle's buffer parity taken from curs.
int enqueue_group_stage(mcv_group *g, const std::vector<mcv_handle *> &act, const std::vector<int> &curs, int s) {
  const StageLauncher &L = act[0]->cands[g->cand];
  StageBatch<kMaxGrids> b;
  std::memset(&b, 0, sizeof(b));
  for (size_t k = 0; k < act.size(); ++k)
    if (int rc = add_grid(b, (int)k, act[k], L, s, curs[k])) return rc;
  number_items(b, (int)act.size());
  const int ctas = std::max(1, std::min(b.total, g->bps * act[0]->nsm));
  L.launch_batch[stage_kind(act[0], s)](dim3(ctas), g->stream, b, true);
  launch_halo_batch<kMaxGrids>(act.data(), curs.data(), (int)act.size(), s, g->stream);
  return MCV_OK;
}

int build_group_graphs(mcv_group *g, const std::vector<mcv_handle *> &act) {
  drop_group_graphs(g);
  std::vector<int> curs(act.size());
  for (size_t k = 0; k < act.size(); ++k) curs[k] = act[k]->mixed ? act[k]->cur : 0;
  const bool mixed = act[0]->mixed;
  for (int c = 0; c < (mixed ? 2 : 1); ++c) {
    MCV_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal), "begin group capture");
    int rc = MCV_OK;
    for (int s = 0; s < num_stages(act[0]) && !rc; ++s) rc = enqueue_group_stage(g, act, curs, s);
    cudaError_t le = cudaGetLastError();
    cudaGraph_t graph = nullptr;
    cudaError_t ce = cudaStreamEndCapture(g->stream, &graph);
    if (rc || le != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      return rc ? rc : cuda_fail(le, "launch during group capture");
    }
    MCV_CUDA(ce, "end group capture");
    cudaError_t ie = cudaGraphInstantiate(&g->graph[c], graph, 0);
    cudaGraphDestroy(graph);
    MCV_CUDA(ie, "instantiate group graph");
    for (int &x : curs) x = 1 - x;  // the next step reads the other buffers
  }
  g->key_hs = act;
  g->key_cur.resize(act.size());
  g->key_active.resize(act.size());
  g->key_ident.resize(act.size());
  for (size_t k = 0; k < act.size(); ++k) {
    g->key_cur[k] = act[k]->mixed ? act[k]->cur : 0;
    g->key_active[k] = act[k]->n_active;
    g->key_ident[k] = act[k]->active_ident;
  }
  return MCV_OK;
}

// The handles a group step advances (those with active members) and the step
// graph to replay first (0, or 1 when the parities are one step on), rebuilt
// unless the handles, active counts, identity of the active lists and buffer
// parities are the ones the graphs were built for.
int prepare_group(mcv_group *g, std::vector<mcv_handle *> &act, int &flip) {
  act.clear();
  for (mcv_handle *h : g->hs) {
    bool idle = false;
    if (int rc = ready_to_step(h, &idle)) return rc;
    if (!idle) act.push_back(h);
  }
  flip = 0;
  if (act.empty()) return MCV_OK;
  bool same = g->graph[0] && g->key_hs == act;
  if (same) {
    int eq = 1, cp = 1;
    for (size_t k = 0; k < act.size(); ++k) {
      const int c = act[k]->mixed ? act[k]->cur : 0;
      same = same && g->key_active[k] == act[k]->n_active && g->key_ident[k] == (int)act[k]->active_ident;
      eq = eq && c == g->key_cur[k];
      cp = cp && c == 1 - g->key_cur[k];
    }
    same = same && (eq || (cp && act[0]->mixed));
    flip = eq ? 0 : 1;
  }
  if (!same) {
    flip = 0;
    return build_group_graphs(g, act);
  }
  return MCV_OK;
}

}  // namespace

extern "C" int mcv_group_create(mcv_handle *const *handles, int count, int tile, mcv_group **out) {
  if (!out) return fail(MCV_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!handles || count < 1 || count > kMaxGrids) return fail(MCV_ERR_ARG, "a group holds 1..4 handles");
  for (int k = 0; k < count; ++k) {
    const mcv_handle *h = handles[k];
    if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
    for (int j = 0; j < k; ++j)
      if (handles[j] == h) return fail(MCV_ERR_ARG, "a handle is listed twice");
    if (h->order != handles[0]->order || h->precision != handles[0]->precision ||
        h->scheme != handles[0]->scheme || h->device != handles[0]->device)
      return fail(MCV_ERR_ARG, "the handles of a group share order, precision, scheme and device");
  }
  const int cand = tile >= 0 ? tile : handles[0]->choice;
  if (cand < 0 || cand >= handles[0]->ncands || !handles[0]->cands[cand].tma)
    return fail(MCV_ERR_ARG, "the group's stage-kernel candidate must be a persistent TMA form (mcv_tuning)");
  mcv_group *g = new mcv_group();
  g->hs.assign(handles, handles + count);
  g->cand = cand;
  g->bps = handles[0]->bps[cand];
  cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
  g->ready.assign(count, nullptr);
  for (int k = 0; k < count && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&g->ready[k], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    mcv_group_destroy(g);
    return cuda_fail(e, "group stream and events");
  }
  *out = g;
  return MCV_OK;
}

extern "C" int mcv_group_step_async(mcv_group *g, int nsteps) {
  if (!g) return fail(MCV_ERR_ARG, "group is NULL");
  if (nsteps < 0) return fail(MCV_ERR_ARG, "nsteps must be >= 0");
  std::vector<mcv_handle *> act;
  int flip = 0;
  if (int rc = prepare_group(g, act, flip)) return rc;
  if (act.empty() || nsteps == 0) return MCV_OK;
  // the group's stream runs after the work already queued on every handle's stream
  for (size_t k = 0; k < g->hs.size(); ++k) {
    MCV_CUDA(cudaEventRecord(g->ready[k], g->hs[k]->stream), "record handle event");
    MCV_CUDA(cudaStreamWaitEvent(g->stream, g->ready[k], 0), "order group after handle");
  }
  int c = flip;
  for (int it = 0; it < nsteps; ++it) {
    MCV_CUDA(cudaGraphLaunch(g->graph[c], g->stream), "launch group graph");
    if (act[0]->mixed) c = 1 - c;
  }
  // and every handle's later work runs after the group's
  MCV_CUDA(cudaEventRecord(g->done, g->stream), "record group event");
  for (mcv_handle *h : g->hs) MCV_CUDA(cudaStreamWaitEvent(h->stream, g->done, 0), "order handle after group");
  for (mcv_handle *h : act) {
    if (h->mixed && (nsteps % 2)) h->cur = 1 - h->cur;
    for (int k = 0; k < h->n_active; ++k) {
      const int m = h->active_host[k];
      h->steps_done[m] += nsteps;
      if (h->mixed) h->mcur[m] = h->cur;
    }
  }
  return MCV_OK;
}

extern "C" int mcv_group_sync(mcv_group *g) {
  if (!g) return fail(MCV_ERR_ARG, "group is NULL");
  MCV_CUDA(cudaStreamSynchronize(g->stream), "group step");
  for (mcv_handle *h : g->hs)
    if (int rc = mcv_sync(h)) return rc;
  return MCV_OK;
}

extern "C" int mcv_group_step(mcv_group *g, int nsteps) {
  if (int rc = mcv_group_step_async(g, nsteps)) return rc;
  return mcv_group_sync(g);
}

extern "C" int mcv_group_query(mcv_group *g) {
  if (!g) return fail(MCV_ERR_ARG, "group is NULL");
  const cudaError_t e = cudaStreamQuery(g->stream);
  if (e == cudaSuccess) return MCV_OK;
  if (e == cudaErrorNotReady) {
    cudaGetLastError();
    return MCV_BUSY;
  }
  return cuda_fail(e, "group query");
}

extern "C" int mcv_group_time_steps(mcv_group *g, int nsteps, double *ms) {
  if (!g || nsteps < 1 || !ms) return fail(MCV_ERR_ARG, "group, nsteps >= 1 and ms required");
  // graphs built and earlier work on the handles' streams done before timing
  std::vector<mcv_handle *> act;
  int flip = 0;
  if (int rc = prepare_group(g, act, flip)) return rc;
  for (mcv_handle *h : g->hs) MCV_CUDA(cudaStreamSynchronize(h->stream), "drain handle before timing");
  cudaEvent_t e0, e1;
  MCV_CUDA(cudaEventCreate(&e0), "event");
  MCV_CUDA(cudaEventCreate(&e1), "event");
  cudaEventRecord(e0, g->stream);
  int rc = mcv_group_step_async(g, nsteps);
  cudaEventRecord(e1, g->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "timed group steps");
  *ms = t;
  return mcv_group_sync(g);
}

extern "C" int mcv_group_destroy(mcv_group *g) {
  if (!g) return MCV_OK;
  if (g->stream) cudaStreamSynchronize(g->stream);
  drop_group_graphs(g);
  for (cudaEvent_t e : g->ready)
    if (e) cudaEventDestroy(e);
  if (g->done) cudaEventDestroy(g->done);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
  return MCV_OK;
}
