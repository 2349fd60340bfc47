// server_host_test.cpp -- the native request loop (mcv_server.cpp, unchanged)
// against fake handles (fake_handles.cpp): every forecast gets exactly its
// steps and its own initial state, slots are reused, pools of other grids
// wait for budget and evict idle empty pools, and no handle is touched while
// it has a chunk queued.  Prints "ok" or the first failed check.
#include <cstdio>
#include <map>
#include <vector>

#include "../../include/mcv_gpu.h"

extern int g_live_handles;
extern long long g_created;
extern int g_live_groups;
extern long long g_group_steps;

#define CHECK(c)                                              \
  do {                                                        \
    if (!(c)) {                                               \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #c); \
      return 1;                                               \
    }                                                         \
  } while (0)

struct Expect {
  double seed;
  long long nsteps;
  int npx;
};

// Polls until every expected forecast is back; checks each result exactly.
static int drain(mcv_server *s, std::map<long long, Expect> &want, long long *stats_out) {
  for (int iter = 0; iter < 200000 && !want.empty(); ++iter) {
    long long ids[4];
    int n = 0;
    CHECK(mcv_server_poll(s, ids, 4, &n) == MCV_OK);
    for (int k = 0; k < n; ++k) {
      auto it = want.find(ids[k]);
      CHECK(it != want.end());
      const size_t sz = (size_t)it->second.npx * it->second.npx * 6;
      std::vector<double> u(sz), v(sz);
      long long steps = -1;
      int finite = -1;
      CHECK(mcv_server_result(s, ids[k], u.data(), v.data(), nullptr, nullptr, &steps, &finite) == MCV_OK);
      CHECK(u[0] == it->second.seed && u[sz - 1] == it->second.seed);
      CHECK(v[0] == (double)it->second.nsteps && steps == it->second.nsteps && finite == 1);
      CHECK(mcv_server_result(s, ids[k], nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == MCV_ERR_ARG);
      want.erase(it);
    }
  }
  CHECK(want.empty());
  CHECK(mcv_server_stats(s, stats_out) == MCV_OK);
  return 0;
}

static int npx_of(int order, int nc) {
  int npx, n, h;
  mcv_grid_sizes(order, nc, &npx, &n, &h);
  return npx;
}

static int submit_host(mcv_server *s, int order, int nc, double dt, long long nsteps, double seed,
                       std::map<long long, Expect> &want) {
  const int npx = npx_of(order, nc);
  std::vector<double> f((size_t)npx * npx * 6, seed);
  long long id = 0;
  CHECK(mcv_server_submit(s, order, nc, dt, nsteps, f.data(), f.data(), f.data(), f.data(), &id) == MCV_OK);
  want[id] = Expect{seed, nsteps, npx};
  return 0;
}

static int submit_spec(mcv_server *s, int order, int nc, double dt, long long nsteps, double gh0,
                       std::map<long long, Expect> &want) {
  long long id = 0;
  CHECK(mcv_server_submit_balanced_flow(s, order, nc, dt, nsteps, gh0, 0., 0., 0, nullptr, 0., 0., 0., 0., 0., &id) ==
        MCV_OK);
  want[id] = Expect{gh0, nsteps, npx_of(order, nc)};
  return 0;
}

int main() {
  long long st[9];
  {
    // three grids (the third differs from the first only in dt), host-array
    // and spec requests, more requests than slots
    mcv_server *s = nullptr;
    CHECK(mcv_server_create(MCV_MIXED, MCV_RK3_TVD, 6.371e6, 1LL << 40, 2400, 32, 0.1, -1, &s) == MCV_OK);
    std::map<long long, Expect> want;
    CHECK(mcv_server_prepare(s, 3, 4, 100.) == MCV_OK);
    const long long created0 = g_created;
    CHECK(mcv_server_prepare(s, 3, 4, 100.) == MCV_OK && g_created == created0);  // the grid's pool exists
    const int steps[] = {7, 1, 23, 4, 12, 9, 3, 17};
    for (int i = 0; i < 8; ++i) {
      const int grid = i % 3;
      const int order = grid == 1 ? 4 : 3;
      const double dt = grid == 2 ? 200. : (grid == 1 ? 50. : 100.);
      if (i % 2) {
        CHECK(submit_spec(s, order, 4, dt, steps[i], 1000. + i, want) == 0);
      } else {
        CHECK(submit_host(s, order, 4, dt, steps[i], 100. + i, want) == 0);
      }
    }
    long long waiting_id = 0;
    {
      const int npx = npx_of(3, 4);
      std::vector<double> f((size_t)npx * npx * 6, 5.);
      CHECK(mcv_server_submit(s, 3, 4, 100., 2, f.data(), f.data(), f.data(), f.data(), &waiting_id) == MCV_OK);
      CHECK(mcv_server_result(s, waiting_id, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == MCV_BUSY);
      want[waiting_id] = Expect{5., 2, npx};
    }
    CHECK(drain(s, want, st) == 0);
    CHECK(st[0] == 0 && st[1] == 0 && st[2] == 0);  // nothing waiting, running or unclaimed
    CHECK(st[6] >= 3 && st[7] == 0);                // one pool per grid at least, no eviction
    CHECK(mcv_server_destroy(s) == MCV_OK);
    CHECK(g_live_handles == 0);
  }
  {
    // a budget that holds one pool at a time: the requests of the first grid
    // that fit are served first, then its pool, idle and empty, is evicted
    // for the other grid's
    mcv_server *s = nullptr;
    CHECK(mcv_server_create(MCV_FP64, MCV_RK4, 6.371e6, 3500, 2400, 32, 0.1, 0, &s) == MCV_OK);
    std::map<long long, Expect> want;
    for (int i = 0; i < 6; ++i) CHECK(submit_host(s, i % 2 ? 4 : 3, 4, 60., 3 + 2 * i, 10. + i, want) == 0);
    CHECK(drain(s, want, st) == 0);
    CHECK(st[6] == 2 && st[7] == 1 && st[3] == 1);  // two pools created, one evicted, one left
    CHECK(mcv_server_destroy(s) == MCV_OK);
    CHECK(g_live_handles == 0);
  }
  {
    // a grid whose one-slot pool exceeds the budget is refused at submission
    mcv_server *s = nullptr;
    CHECK(mcv_server_create(MCV_FP64, MCV_RK4, 6.371e6, 1500, 2400, 32, 0.1, -1, &s) == MCV_OK);
    std::map<long long, Expect> want;
    const int npx = npx_of(4, 4);
    std::vector<double> f((size_t)npx * npx * 6, 1.);
    long long id;
    CHECK(mcv_server_submit(s, 4, 4, 60., 2, f.data(), f.data(), f.data(), f.data(), &id) == MCV_ERR_NOMEM);
    CHECK(mcv_server_destroy(s) == MCV_OK);
  }
  {
    // slot_bytes allows 32 slots but the budget holds one member: the pool is
    // made with the slots the budget holds, and every request is served
    // (2200 bytes for one member of (3, 4) with the fake footprint, 3400 for two)
    mcv_server *s = nullptr;
    CHECK(mcv_server_create(MCV_FP64, MCV_RK4, 6.371e6, 2500, 1LL << 30, 32, 0.1, -1, &s) == MCV_OK);
    std::map<long long, Expect> want;
    for (int i = 0; i < 3; ++i) CHECK(submit_host(s, 3, 4, 60., 2 + i, 20. + i, want) == 0);
    CHECK(drain(s, want, st) == 0);
    CHECK(st[6] == 1 && st[5] == 2200);  // one pool of one slot
    CHECK(mcv_server_destroy(s) == MCV_OK);
    CHECK(g_live_handles == 0);
  }
  {
    // a request whose initial state is refused and one whose read-back fails
    // are retired as failed (their result calls return the error, once); the
    // poll reports each error and the other forecasts still finish
    mcv_server *s = nullptr;
    CHECK(mcv_server_create(MCV_MIXED, MCV_RK3_TVD, 6.371e6, 1LL << 40, 2400, 32, 0.1, -1, &s) == MCV_OK);
    std::map<long long, Expect> want;
    long long bad_spec = 0, bad_read = 0;
    CHECK(mcv_server_submit_balanced_flow(s, 3, 4, 100., 5, -1., 0., 0., 0, nullptr, 0., 0., 0., 0., 0., &bad_spec) ==
          MCV_OK);
    {
      const int npx = npx_of(3, 4);
      std::vector<double> f((size_t)npx * npx * 6, 666.);
      CHECK(mcv_server_submit(s, 3, 4, 100., 3, f.data(), f.data(), f.data(), f.data(), &bad_read) == MCV_OK);
    }
    for (int i = 0; i < 4; ++i) CHECK(submit_host(s, 3, 4, 100., 4 + i, 30. + i, want) == 0);
    int errors = 0;
    bool got_spec = false, got_read = false;
    for (int iter = 0; iter < 200000 && (!want.empty() || !got_spec || !got_read); ++iter) {
      long long ids[4];
      int n = 0;
      const int rc = mcv_server_poll(s, ids, 4, &n);
      if (rc != MCV_OK) ++errors;
      for (int k = 0; k < n; ++k) {
        if (ids[k] == bad_spec || ids[k] == bad_read) {
          long long steps = -1;
          int finite = -1;
          const int want_rc = ids[k] == bad_spec ? MCV_ERR_ARG : MCV_ERR_CUDA;
          CHECK(mcv_server_result(s, ids[k], nullptr, nullptr, nullptr, nullptr, &steps, &finite) == want_rc);
          CHECK(finite == 0 && steps == (ids[k] == bad_spec ? 5 : 3));
          CHECK(mcv_server_result(s, ids[k], nullptr, nullptr, nullptr, nullptr, nullptr, nullptr) == MCV_ERR_ARG);
          (ids[k] == bad_spec ? got_spec : got_read) = true;
          continue;
        }
        auto it = want.find(ids[k]);
        CHECK(it != want.end());
        const size_t sz = (size_t)it->second.npx * it->second.npx * 6;
        std::vector<double> u(sz), v(sz);
        long long steps = -1;
        int finite = -1;
        CHECK(mcv_server_result(s, ids[k], u.data(), v.data(), nullptr, nullptr, &steps, &finite) == MCV_OK);
        CHECK(u[0] == it->second.seed && v[0] == (double)it->second.nsteps && finite == 1);
        want.erase(it);
      }
    }
    CHECK(want.empty() && got_spec && got_read && errors == 2);
    CHECK(mcv_server_stats(s, st) == MCV_OK);
    CHECK(st[0] == 0 && st[1] == 0 && st[2] == 0);
    CHECK(mcv_server_destroy(s) == MCV_OK);
    CHECK(g_live_handles == 0);
  }
  {
    // grouping: pools of one order with close step costs advance together in
    // one group chunk; every forecast still gets exactly its steps
    mcv_server *s = nullptr;
    CHECK(mcv_server_create(MCV_MIXED, MCV_RK3_TVD, 6.371e6, 1LL << 40, 2400, 32, 0.1, 0, &s) == MCV_OK);
    long long gc = -1;
    CHECK(mcv_server_set_grouping(s, 0, 2., &gc) == MCV_ERR_ARG);
    CHECK(mcv_server_set_grouping(s, 3, 4., &gc) == MCV_OK && gc == 0);
    std::map<long long, Expect> want;
    const int ncs[] = {4, 5, 6, 4, 5, 6, 5, 4};
    const long long steps[] = {9, 4, 13, 2, 7, 5, 11, 3};
    for (int i = 0; i < 8; ++i) CHECK(submit_host(s, 3, ncs[i], 100., steps[i], 50. + i, want) == 0);
    CHECK(submit_host(s, 4, 4, 100., 6, 70., want) == 0);  // another order: never grouped with the others
    const long long group_steps0 = g_group_steps;
    CHECK(drain(s, want, st) == 0);
    CHECK(g_group_steps > group_steps0);
    CHECK(mcv_server_set_grouping(s, 3, 4., &gc) == MCV_OK && gc == g_group_steps - group_steps0);
    CHECK(mcv_server_destroy(s) == MCV_OK);
    CHECK(g_live_handles == 0 && g_live_groups == 0);
  }
  std::printf("ok\n");
  return 0;
}
