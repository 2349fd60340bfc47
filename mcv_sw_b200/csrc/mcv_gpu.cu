// mcv_gpu.cu -- C ABI (include/mcv_gpu.h) over the sm_100a kernels.
//
// A handle holds one grid (order, Nc) and `members` states, all resident in
// HBM.  One RK step is 2 * stages kernel launches (fused stage K1, halo K2),
// captured once into a CUDA graph and replayed per step.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mcv_gpu.h"
#include "mcv_internal.h"
#include "mcv_kernels.cuh"

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

#define MCV_CUDA(call, what)                      \
  do {                                            \
    cudaError_t _e = (call);                      \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

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

// Tile shapes (cells) of the stage kernel per order.
template <int D>
struct TileShape;
template <>
struct TileShape<3> {
  static constexpr int CX = 12, CY = 12, NT = 320;
};
template <>
struct TileShape<4> {
  static constexpr int CX = 8, CY = 8, NT = 320;
};

}  // namespace mcv

using namespace mcv;

struct mcv_handle {
  int order = 0, nc = 0, scheme = 0, precision = 0, members = 0;
  double dt = 0, radius = 0;
  GridDesc g{};
  int H = 0, npx = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  // device memory (one allocation)
  void *pool = nullptr;
  size_t pool_bytes = 0;
  double *Y[3]{}, *A[3]{}, *B[3]{}, *acc[3]{};
  double *sqrtG = nullptr, *ig11 = nullptr, *ig12 = nullptr, *ig22 = nullptr, *fcor = nullptr, *phis = nullptr;
  double4 *bnd = nullptr, *Mtab = nullptr, *Ntab = nullptr;
  int *giref = nullptr;
  double2 *gcoef = nullptr;
  double4 *partial = nullptr;
  double dx2 = 0, dx3 = 0;
  bool geometry_set = false;
  std::vector<char> member_set;
  std::vector<long long> steps_done;
  std::vector<double> sqrtG_host;  // padded Fortran layout, for phiG on download
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
};

namespace {

constexpr int kPartialBlocks = 296;

struct Layout {
  size_t field;   // bytes of one padded field for all members
  size_t plane6;  // bytes of one padded field of one member (6 panels)
  size_t total;
  size_t off_state[9], off_acc[3], off_metric[5], off_phis, off_bnd, off_M, off_N, off_iref, off_coef, off_partial;
};

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

Layout make_layout(const GridDesc &g, int H, int scheme, int members) {
  Layout L{};
  L.plane6 = (size_t)g.mstride * sizeof(double);
  L.field = L.plane6 * members;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes, 256);
    return o;
  };
  for (int k = 0; k < 9; ++k) L.off_state[k] = take(L.field);
  for (int k = 0; k < 3; ++k) L.off_acc[k] = (scheme == MCV_RK4) ? take(L.field) : 0;
  for (int k = 0; k < 5; ++k) L.off_metric[k] = take(L.plane6);
  L.off_phis = take(L.field);
  L.off_bnd = take(sizeof(double4) * 24 * (size_t)g.n * members);
  L.off_M = take(sizeof(double4) * 24 * (size_t)(H + 1) * g.n);
  L.off_N = take(sizeof(double4) * 24 * (size_t)(H + 1) * g.n);
  L.off_iref = take(sizeof(int) * (size_t)H * g.n);
  L.off_coef = take(sizeof(double2) * (size_t)H * g.n);
  L.off_partial = take(sizeof(double4) * kPartialBlocks);
  L.total = off;
  return L;
}

// Copy a host array in the reference's padded Fortran layout (npx*npx*6,
// contiguous) into the pitched device layout of member slot `dst`.
int upload_padded(mcv_handle *h, double *dst, const double *src) {
  const size_t row = (size_t)h->npx * sizeof(double);
  MCV_CUDA(cudaMemcpy2DAsync(dst, (size_t)h->g.P * sizeof(double), src, row, row, (size_t)h->npx * 6,
                             cudaMemcpyHostToDevice, h->stream),
           "upload field");
  return MCV_OK;
}

int download_padded(mcv_handle *h, double *dst, const double *src) {
  const size_t row = (size_t)h->npx * sizeof(double);
  MCV_CUDA(cudaMemcpy2DAsync(dst, row, src, (size_t)h->g.P * sizeof(double), row, (size_t)h->npx * 6,
                             cudaMemcpyDeviceToHost, h->stream),
           "download field");
  return MCV_OK;
}

template <int D, int KIND>
void launch_stage(mcv_handle *h, const StageArgs &a) {
  using S = TileShape<D>;
  using T = Tile<D, S::CX, S::CY>;
  dim3 grid(h->g.tiles_x * h->g.tiles_y, 6, h->members);
  stage_kernel<D, S::CX, S::CY, S::NT, KIND><<<grid, S::NT, T::BYTES, h->stream>>>(h->g, a);
}

template <int D>
int prepare_kernels() {
  using S = TileShape<D>;
  using T = Tile<D, S::CX, S::CY>;
  const int bytes = (int)T::BYTES;
#define SET_SMEM(KIND)                                                                                         \
  MCV_CUDA(cudaFuncSetAttribute(stage_kernel<D, S::CX, S::CY, S::NT, KIND>,                                 \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),                       \
           "set stage kernel shared memory")
  SET_SMEM(RK3_S1);
  SET_SMEM(RK3_S2);
  SET_SMEM(RK3_S3);
  SET_SMEM(RK4_S1);
  SET_SMEM(RK4_S2);
  SET_SMEM(RK4_S3);
  SET_SMEM(RK4_S4);
#undef SET_SMEM
  return MCV_OK;
}

template <int D>
void launch_halo(mcv_handle *h, double *const st[3]) {
  HaloArgs a{};
  a.u = st[0];
  a.v = st[1];
  a.phi = st[2];
  a.bnd = h->bnd;
  a.Mtab = h->Mtab;
  a.Ntab = h->Ntab;
  a.giref = h->giref;
  a.gcoef = h->gcoef;
  a.dx = h->g.dx;
  a.dx2 = h->dx2;
  a.dx3 = h->dx3;
  a.members = h->members;
  const long long threads = 24LL * (h->H + 1) * h->g.n * h->members;
  const int block = 128;
  halo_kernel<D><<<(unsigned)((threads + block - 1) / block), block, 0, h->stream>>>(h->g, a);
}

StageArgs stage_args(mcv_handle *h, double *const in[3], double *const base[3], double *const out[3], double inc) {
  StageArgs a{};
  a.us = in[0]; a.vs = in[1]; a.ps = in[2];
  a.u0 = base[0]; a.v0 = base[1]; a.p0 = base[2];
  a.uo = out[0]; a.vo = out[1]; a.po = out[2];
  a.aU = h->acc[0]; a.aV = h->acc[1]; a.aP = h->acc[2];
  a.sqrtG = h->sqrtG; a.ig11 = h->ig11; a.ig12 = h->ig12; a.ig22 = h->ig22; a.fcor = h->fcor;
  a.phis = h->phis;
  a.bnd = h->bnd;
  a.inc = inc;
  return a;
}

// Stage s of one RK step on every member (the stage sequence of RK3_TVD /
// RK4, src/time_scheme_mod.F90:13-69): the fused stage kernel, then the halo
// kernel on the stage's output.
template <int D>
void enqueue_stage(mcv_handle *h, int s, cudaEvent_t mid = nullptr) {
  const double dt = h->dt;
  double *const *out = nullptr;
  if (h->scheme == MCV_RK3_TVD) {
    switch (s) {
      case 0: launch_stage<D, RK3_S1>(h, stage_args(h, h->Y, h->Y, h->A, dt)); out = h->A; break;
      case 1: launch_stage<D, RK3_S2>(h, stage_args(h, h->A, h->Y, h->B, 0.25 * dt)); out = h->B; break;
      default: launch_stage<D, RK3_S3>(h, stage_args(h, h->B, h->Y, h->Y, 2. / 3. * dt)); out = h->Y; break;
    }
  } else {
    switch (s) {
      case 0: launch_stage<D, RK4_S1>(h, stage_args(h, h->Y, h->Y, h->A, 0.5 * dt)); out = h->A; break;
      case 1: launch_stage<D, RK4_S2>(h, stage_args(h, h->A, h->Y, h->B, 0.5 * dt)); out = h->B; break;
      case 2: launch_stage<D, RK4_S3>(h, stage_args(h, h->B, h->Y, h->A, dt)); out = h->A; break;
      default: launch_stage<D, RK4_S4>(h, stage_args(h, h->A, h->Y, h->Y, dt)); out = h->Y; break;
    }
  }
  if (mid) cudaEventRecord(mid, h->stream);
  launch_halo<D>(h, out);
}

int num_stages(const mcv_handle *h) { return h->scheme == MCV_RK3_TVD ? 3 : 4; }

void enqueue_stage_any(mcv_handle *h, int s, cudaEvent_t mid = nullptr) {
  if (h->order == 3) enqueue_stage<3>(h, s, mid);
  else enqueue_stage<4>(h, s, mid);
}

void enqueue_step(mcv_handle *h) {
  for (int s = 0; s < num_stages(h); ++s) enqueue_stage_any(h, s);
}

int build_graph(mcv_handle *h) {
  if (h->graph_exec) return MCV_OK;
  MCV_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal), "begin step capture");
  enqueue_step(h);
  cudaError_t le = cudaGetLastError();
  cudaGraph_t graph = nullptr;
  cudaError_t ce = cudaStreamEndCapture(h->stream, &graph);
  if (le != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    return cuda_fail(le, "launch during step capture");
  }
  MCV_CUDA(ce, "end step capture");
  h->graph = graph;
  MCV_CUDA(cudaGraphInstantiate(&h->graph_exec, graph, 0), "instantiate step graph");
  return MCV_OK;
}

}  // namespace

extern "C" const char *mcv_last_error(void) { return g_last_error.c_str(); }

extern "C" long long mcv_footprint_bytes(int order, int nc, int scheme, int precision, int members) {
  if ((order != 3 && order != 4) || nc < 2 || members < 1) return -1;
  (void)precision;
  GridDesc g{};
  int H, npx;
  grid_desc(order, nc, g, H, npx);
  return (long long)make_layout(g, H, scheme, members).total;
}

extern "C" int mcv_create(int order, int nc, int scheme, int precision, double dt, double radius, int members,
                          mcv_handle **out) {
  if (!out) return fail(MCV_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (order != 3 && order != 4) return fail(MCV_ERR_ARG, "order must be 3 (MCV3) or 4 (MCV4)");
  if (nc < 2 || nc > 4096) return fail(MCV_ERR_ARG, "nc out of range [2, 4096]");
  if (scheme != MCV_RK3_TVD && scheme != MCV_RK4) return fail(MCV_ERR_ARG, "scheme must be MCV_RK3_TVD or MCV_RK4");
  if (precision != MCV_FP64) return fail(MCV_ERR_ARG, "precision not supported by this build");
  if (!(dt > 0) || !std::isfinite(dt)) return fail(MCV_ERR_ARG, "dt must be positive and finite");
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

  mcv_handle *h = new mcv_handle();
  h->order = order; h->nc = nc; h->scheme = scheme; h->precision = precision; h->members = members;
  h->dt = dt; h->radius = radius; h->device = dev;
  grid_desc(order, nc, h->g, h->H, h->npx);
  const double pi = 2.0 * std::asin(1.0);
  h->g.dx = (90. / nc) * (pi / 180.);
  h->g.inv_dx = 1. / h->g.dx;
  h->g.inv_2dx = 1. / (2. * h->g.dx);
  h->g.inv_dx2 = 1. / (h->g.dx * h->g.dx);
  h->dx2 = h->g.dx * h->g.dx;
  h->dx3 = std::pow(h->g.dx, 3.);
  int CX = order == 3 ? TileShape<3>::CX : TileShape<4>::CX, CY = order == 3 ? TileShape<3>::CY : TileShape<4>::CY;
  h->g.tiles_x = (nc + CX - 1) / CX;
  h->g.tiles_y = (nc + CY - 1) / CY;
  h->member_set.assign(members, 0);
  h->steps_done.assign(members, 0);

  int rc = upload_tables();
  if (!rc) rc = (order == 3) ? prepare_kernels<3>() : prepare_kernels<4>();
  if (rc) {
    delete h;
    return rc;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete h;
    return cuda_fail(e, "create stream");
  }
  Layout L = make_layout(h->g, h->H, scheme, members);
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
    h->Y[k] = (double *)(base + L.off_state[k]);
    h->A[k] = (double *)(base + L.off_state[3 + k]);
    h->B[k] = (double *)(base + L.off_state[6 + k]);
    h->acc[k] = scheme == MCV_RK4 ? (double *)(base + L.off_acc[k]) : nullptr;
  }
  h->sqrtG = (double *)(base + L.off_metric[0]);
  h->ig11 = (double *)(base + L.off_metric[1]);
  h->ig12 = (double *)(base + L.off_metric[2]);
  h->ig22 = (double *)(base + L.off_metric[3]);
  h->fcor = (double *)(base + L.off_metric[4]);
  h->phis = (double *)(base + L.off_phis);
  h->bnd = (double4 *)(base + L.off_bnd);
  h->Mtab = (double4 *)(base + L.off_M);
  h->Ntab = (double4 *)(base + L.off_N);
  h->giref = (int *)(base + L.off_iref);
  h->gcoef = (double2 *)(base + L.off_coef);
  h->partial = (double4 *)(base + L.off_partial);
  // zero everything once: unused pitch padding and halo corners stay finite
  e = cudaMemsetAsync(h->pool, 0, L.total, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    int r = cuda_fail(e, "clear device memory");
    mcv_destroy(h);
    return r;
  }
  (void)radius;
  *out = h;
  return MCV_OK;
}

extern "C" int mcv_destroy(mcv_handle *h) {
  if (!h) return MCV_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
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
    g11[k] = matrixIG[4 * k + 0];
    g12[k] = matrixIG[4 * k + 2];  // IG(1,2) == IG(2,1) (projection_mod.F90:186)
    g22[k] = matrixIG[4 * k + 3];
  }
  for (size_t k = 0; k < NP; ++k)
    if (matrixIG[4 * k + 1] != matrixIG[4 * k + 2]) return fail(MCV_ERR_ARG, "matrixIG is not symmetric");
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
  int rc;
  if ((rc = upload_padded(h, h->sqrtG, sqrtG))) return rc;
  if ((rc = upload_padded(h, h->ig11, g11.data()))) return rc;
  if ((rc = upload_padded(h, h->ig12, g12.data()))) return rc;
  if ((rc = upload_padded(h, h->ig22, g22.data()))) return rc;
  if ((rc = upload_padded(h, h->fcor, f))) return rc;
  MCV_CUDA(cudaMemcpyAsync(h->Mtab, Mt.data(), Mt.size() * sizeof(double4), cudaMemcpyHostToDevice, h->stream), "upload Mtab");
  MCV_CUDA(cudaMemcpyAsync(h->Ntab, Nt.data(), Nt.size() * sizeof(double4), cudaMemcpyHostToDevice, h->stream), "upload Ntab");
  MCV_CUDA(cudaMemcpyAsync(h->giref, ghost_iref, sizeof(int) * (size_t)H * n, cudaMemcpyHostToDevice, h->stream), "upload iref");
  MCV_CUDA(cudaMemcpyAsync(h->gcoef, coef.data(), sizeof(double2) * coef.size(), cudaMemcpyHostToDevice, h->stream), "upload coef");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "geometry upload");
  h->sqrtG_host.assign(sqrtG, sqrtG + NP);
  h->geometry_set = true;
  return MCV_OK;
}

extern "C" int mcv_set_member(mcv_handle *h, int m, const double *phi_s, const double *u, const double *v,
                              const double *phi) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (m < 0 || m >= h->members) return fail(MCV_ERR_ARG, "member index out of range");
  if (!phi_s || !u || !v || !phi) return fail(MCV_ERR_ARG, "state array is NULL");
  const long long off = (long long)m * h->g.mstride;
  int rc;
  if ((rc = upload_padded(h, h->phis + off, phi_s))) return rc;
  if ((rc = upload_padded(h, h->Y[0] + off, u))) return rc;
  if ((rc = upload_padded(h, h->Y[1] + off, v))) return rc;
  if ((rc = upload_padded(h, h->Y[2] + off, phi))) return rc;
  MCV_CUDA(cudaStreamSynchronize(h->stream), "member upload");
  h->member_set[m] = 1;
  h->steps_done[m] = 0;
  return MCV_OK;
}

extern "C" int mcv_step_async(mcv_handle *h, int nsteps) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (nsteps < 0) return fail(MCV_ERR_ARG, "nsteps must be >= 0");
  if (!h->geometry_set) return fail(MCV_ERR_ORDER, "mcv_set_geometry must precede mcv_step");
  for (int m = 0; m < h->members; ++m)
    if (!h->member_set[m]) return fail(MCV_ERR_ORDER, "every member must be set before mcv_step");
  if (int rc = build_graph(h)) return rc;
  for (int s = 0; s < nsteps; ++s) MCV_CUDA(cudaGraphLaunch(h->graph_exec, h->stream), "launch step graph");
  for (int m = 0; m < h->members; ++m) h->steps_done[m] += nsteps;
  return MCV_OK;
}

extern "C" int mcv_sync(mcv_handle *h) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  MCV_CUDA(cudaStreamSynchronize(h->stream), "step");
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
  int rc;
  if (u && (rc = download_padded(h, u, h->Y[0] + off))) return rc;
  if (v && (rc = download_padded(h, v, h->Y[1] + off))) return rc;
  if (phi_dst && (rc = download_padded(h, phi_dst, h->Y[2] + off))) return rc;
  MCV_CUDA(cudaStreamSynchronize(h->stream), "state download");
  if (phi_dst && h->steps_done[m] > 0) {
    // halo corners hold FillValue after correct_bdy_ghost (ghost_mod.f90:161,179)
    const int npx = h->npx, H = h->H;
    for (int p = 0; p < 6; ++p)
      for (int j = 0; j < npx; ++j)
        for (int i = 0; i < npx; ++i) {
          const bool xh = i < H || i >= npx - H, yh = j < H || j >= npx - H;
          if (xh && yh) phi_dst[(size_t)i + (size_t)npx * ((size_t)j + (size_t)npx * p)] = -9999999999999999.;
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
  if (h->order == 3)
    mass_energy_kernel<3><<<kPartialBlocks, 256, 0, h->stream>>>(h->g, h->Y[0] + off, h->Y[1] + off, h->Y[2] + off,
                                                                 h->sqrtG, h->ig11, h->ig12, h->ig22, h->phis + off,
                                                                 w0, w1, wden, h->partial);
  else
    mass_energy_kernel<4><<<kPartialBlocks, 256, 0, h->stream>>>(h->g, h->Y[0] + off, h->Y[1] + off, h->Y[2] + off,
                                                                 h->sqrtG, h->ig11, h->ig12, h->ig22, h->phis + off,
                                                                 w0, w1, wden, h->partial);
  MCV_CUDA(cudaGetLastError(), "launch mass/energy");
  std::vector<double4> part(kPartialBlocks);
  MCV_CUDA(cudaMemcpyAsync(part.data(), h->partial, sizeof(double4) * kPartialBlocks, cudaMemcpyDeviceToHost, h->stream),
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

static int ready_to_step(mcv_handle *h) {
  if (!h) return fail(MCV_ERR_ARG, "handle is NULL");
  if (!h->geometry_set) return fail(MCV_ERR_ORDER, "mcv_set_geometry must precede stepping");
  for (int m = 0; m < h->members; ++m)
    if (!h->member_set[m]) return fail(MCV_ERR_ORDER, "every member must be set before stepping");
  return MCV_OK;
}

extern "C" int mcv_time_steps(mcv_handle *h, int nsteps, double *ms) {
  if (int rc = ready_to_step(h)) return rc;
  if (nsteps < 1 || !ms) return fail(MCV_ERR_ARG, "nsteps >= 1 and ms required");
  if (int rc = build_graph(h)) return rc;
  cudaEvent_t e0, e1;
  MCV_CUDA(cudaEventCreate(&e0), "event");
  MCV_CUDA(cudaEventCreate(&e1), "event");
  cudaEventRecord(e0, h->stream);
  for (int s = 0; s < nsteps; ++s) cudaGraphLaunch(h->graph_exec, h->stream);
  cudaEventRecord(e1, h->stream);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_fail(e, "timed steps");
  for (int m = 0; m < h->members; ++m) h->steps_done[m] += nsteps;
  *ms = t;
  return MCV_OK;
}

extern "C" int mcv_profile_step(mcv_handle *h, int nsteps, double *stage_ms, double *halo_ms) {
  if (int rc = ready_to_step(h)) return rc;
  if (nsteps < 1 || !stage_ms || !halo_ms) return fail(MCV_ERR_ARG, "nsteps >= 1 and outputs required");
  const int S = num_stages(h);
  std::vector<cudaEvent_t> ev((size_t)nsteps * S * 3);
  for (auto &e : ev) MCV_CUDA(cudaEventCreate(&e), "event");
  for (int it = 0; it < nsteps; ++it)
    for (int s = 0; s < S; ++s) {
      cudaEvent_t *e = &ev[((size_t)it * S + s) * 3];
      cudaEventRecord(e[0], h->stream);
      enqueue_stage_any(h, s, e[1]);
      cudaEventRecord(e[2], h->stream);
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
  for (int m = 0; m < h->members; ++m) h->steps_done[m] += nsteps;
  return MCV_OK;
}
