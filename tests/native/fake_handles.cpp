// fake_handles.cpp -- stand-ins for the per-handle entry points of
// libmcv_gpu.so, so that mcv_server.cpp (compiled unchanged) runs on a CPU.
// A fake member's "state" records the seed it was loaded with and the steps
// it was advanced: a forecast stepped too far or too little shows up exactly.
// A queued chunk completes after two mcv_query calls.  Two injected failures
// exercise the loop's error paths: a balanced-flow spec with gh0 < 0 is
// refused, and a member loaded with the seed 666 fails its read-back.
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mcv_gpu.h"

namespace mcv {
static std::string g_err;
int fail(int code, const char *msg) {
  g_err = msg;
  return code;
}
}  // namespace mcv

struct mcv_handle {
  int order, nc, members, npx;
  std::vector<double> seed;
  std::vector<long long> steps;
  std::vector<int> active;
  int pending = 0;  // mcv_query calls before the queued chunk completes
  bool geometry = false;
};

int g_live_handles = 0;
long long g_created = 0;

extern "C" {

const char *mcv_last_error(void) { return mcv::g_err.c_str(); }

int mcv_grid_sizes(int order, int nc, int *npx, int *n, int *halo) {
  if ((order != 3 && order != 4) || nc < 2) return mcv::fail(MCV_ERR_ARG, "bad grid");
  *n = nc * (order - 1) + 1;
  *halo = order - 1;
  *npx = *n + 2 * *halo;
  return MCV_OK;
}

long long mcv_footprint_bytes(int order, int nc, int, int, int members) {
  return 1000LL + 100LL * members * order * nc;
}

int mcv_device_memory(long long *free_b, long long *total_b) {
  *free_b = *total_b = 1LL << 40;
  return MCV_OK;
}

int mcv_create(int order, int nc, int, int, double, double, int members, mcv_handle **out) {
  mcv_handle *h = new mcv_handle();
  h->order = order;
  h->nc = nc;
  h->members = members;
  int n, halo;
  mcv_grid_sizes(order, nc, &h->npx, &n, &halo);
  h->seed.assign(members, -1.);
  h->steps.assign(members, 0);
  for (int m = 0; m < members; ++m) h->active.push_back(m);
  *out = h;
  ++g_live_handles;
  ++g_created;
  return MCV_OK;
}

int mcv_set_geometry_equiangular(mcv_handle *h) {
  h->geometry = true;
  return MCV_OK;
}

int mcv_select_tile(mcv_handle *, int) { return MCV_OK; }

int mcv_set_member(mcv_handle *h, int m, const double *phi_s, const double *, const double *, const double *) {
  if (!h->geometry || h->pending) return mcv::fail(MCV_ERR_ORDER, "member set on a busy handle or before geometry");
  h->seed[m] = phi_s[0];
  h->steps[m] = 0;
  return MCV_OK;
}

int mcv_set_member_balanced_flow(mcv_handle *h, int m, double gh0, double, double, int, const double *, double, double,
                                 double, double, double) {
  if (!h->geometry || h->pending) return mcv::fail(MCV_ERR_ORDER, "member set on a busy handle or before geometry");
  if (gh0 < 0.) return mcv::fail(MCV_ERR_ARG, "injected: a spec this fake refuses");
  h->seed[m] = gh0;
  h->steps[m] = 0;
  return MCV_OK;
}

int mcv_set_active(mcv_handle *h, int count, const int *members) {
  if (h->pending) return mcv::fail(MCV_ERR_ORDER, "set_active on a busy handle");
  h->active.assign(members, members + count);
  return MCV_OK;
}

int mcv_step_async(mcv_handle *h, int nsteps) {
  if (h->pending) return mcv::fail(MCV_ERR_ORDER, "step queued on a busy handle");
  for (int m : h->active) h->steps[m] += nsteps;
  h->pending = 2;
  return MCV_OK;
}

int mcv_step(mcv_handle *h, int nsteps) {
  int rc = mcv_step_async(h, nsteps);
  h->pending = 0;
  return rc;
}

int mcv_query(mcv_handle *h) {
  if (h->pending > 0) {
    --h->pending;
    return MCV_BUSY;
  }
  return MCV_OK;
}

int mcv_sync(mcv_handle *h) {
  h->pending = 0;
  return MCV_OK;
}

int mcv_check_finite(mcv_handle *h, int *flags) {
  if (h->pending) return mcv::fail(MCV_ERR_ORDER, "check on a busy handle");
  for (int m = 0; m < h->members; ++m) flags[m] = 0;
  return MCV_OK;
}

int mcv_get_state(mcv_handle *h, int m, double *u, double *v, double *phi, double *phiG) {
  if (h->pending) return mcv::fail(MCV_ERR_ORDER, "download from a busy handle");
  if (h->seed[m] == 666.) return mcv::fail(MCV_ERR_CUDA, "injected: a read-back this fake fails");
  const size_t sz = (size_t)h->npx * h->npx * 6;
  for (size_t k = 0; k < sz; ++k) {
    if (u) u[k] = h->seed[m];
    if (v) v[k] = (double)h->steps[m];
    if (phi) phi[k] = 0.;
    if (phiG) phiG[k] = 0.;
  }
  return MCV_OK;
}

int mcv_destroy(mcv_handle *h) {
  delete h;
  --g_live_handles;
  return MCV_OK;
}

// A fake group steps its handles' active members together; its chunk
// completes after two mcv_group_query calls, during which its handles are busy.
}  // extern "C"
struct mcv_group {
  std::vector<mcv_handle *> hs;
  int pending = 0;
};
int g_live_groups = 0;
long long g_group_steps = 0;
extern "C" {

int mcv_group_create(mcv_handle *const *handles, int count, int, mcv_group **out) {
  if (count < 1 || count > 4) return mcv::fail(MCV_ERR_ARG, "bad group");
  mcv_group *g = new mcv_group();
  g->hs.assign(handles, handles + count);
  *out = g;
  ++g_live_groups;
  return MCV_OK;
}

int mcv_group_step_async(mcv_group *g, int nsteps) {
  for (mcv_handle *h : g->hs)
    if (h->pending) return mcv::fail(MCV_ERR_ORDER, "group step on a busy handle");
  for (mcv_handle *h : g->hs) {
    for (int m : h->active) h->steps[m] += nsteps;
    h->pending = 1000000;  // busy until the group completes
  }
  g->pending = 2;
  ++g_group_steps;
  return MCV_OK;
}

int mcv_group_query(mcv_group *g) {
  if (g->pending > 0 && --g->pending > 0) return MCV_BUSY;
  for (mcv_handle *h : g->hs) h->pending = 0;
  return MCV_OK;
}

int mcv_group_destroy(mcv_group *g) {
  for (mcv_handle *h : g->hs) h->pending = 0;
  delete g;
  --g_live_groups;
  return MCV_OK;
}

}  // extern "C"
