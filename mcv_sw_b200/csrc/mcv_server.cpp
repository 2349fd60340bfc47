// mcv_server.cpp -- continuous-batching forecast server behind the C ABI
// (mcv_server_*).  The reference runs one forecast per process
// (src/MCV_SW.F90); it has no serving layer.  This is the native form of the
// request loop: requests of different order, Nc and length are queued,
// admitted by HBM footprint into member slots of device-resident pools, and
// advanced in chunks of RK steps on the pools' own streams, so pools of
// different grids run on the GPU at the same time.  It is built only on the
// handle entry points of mcv_gpu.h (mcv_create, mcv_set_geometry_equiangular,
// mcv_set_member[_balanced_flow], mcv_set_active, mcv_step_async, mcv_query,
// mcv_check_finite, mcv_get_state), so a request's arithmetic is exactly that
// of a plain handle stepped alone on the same tile shape.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <vector>

#include "../../include/mcv_gpu.h"
#include "mcv_internal.h"

using mcv::fail;

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
  long long id;
  int order, nc;
  double dt;
  long long nsteps;
  bool spec;  // initial state generated on the device from the balanced-flow spec
  std::vector<double> phis, u, v, phi;  // host copies (spec = false)
  double gh0, u0, alpha, rms, mh0, lon_c, lat_c, efold;
  int lmax;
  std::vector<double> coef;
};

struct Finished {
  std::vector<double> u, v, phi, phiG;
  long long nsteps;
  int finite;
  int status = MCV_OK;  // < 0: the forecast failed (admission or read-back); no state
};

struct Pool {
  int order, nc;
  double dt;
  int slots;
  long long bytes;
  mcv_handle *h = nullptr;
  std::vector<long long> req;   // request id held by each slot, -1: free
  std::vector<long long> left;  // steps still to take
  std::vector<long long> total;
  std::vector<int> active;      // slots the next chunk advances
  std::vector<int> dev_active;  // slot list the handle was last given
  bool dev_active_set = false;
  long long in_flight = 0;  // steps of the chunk on the GPU (0: idle)
  double launched = 0.;
  double ms_per_step = -1.;  // measured, or < 0 before the first chunk
  mcv_group *group = nullptr;  // the group whose launch holds the pool's chunk (null: its own stream)

  bool same_grid(int o, int n, double d) const { return order == o && nc == n && dt == d; }
  int free_slot() const {
    for (int s = 0; s < slots; ++s)
      if (req[s] < 0) return s;
    return -1;
  }
  bool empty() const {
    for (long long r : req)
      if (r >= 0) return false;
    return true;
  }
};

}  // namespace

struct mcv_server {
  int precision, scheme, tile, max_slots;
  double radius, chunk_ms;
  long long budget, slot_bytes;
  long long next_id = 1;
  std::deque<Request> waiting;
  std::vector<Pool *> pools;
  std::map<long long, Finished> finished;
  std::deque<long long> unreported;  // finished ids not yet returned by mcv_server_poll
  long long pools_created = 0, pools_evicted = 0, chunks = 0;
  // grouping: idle pools of one order whose per-member step costs fall in one
  // bucket of a log scale of base group_ratio advance together, up to
  // group_max per launch
  int group_max = 1;
  double group_ratio = 1.;
  std::map<std::vector<mcv_handle *>, mcv_group *> groups;  // cached groups by pool handles
  long long grouped_chunks = 0;
};

namespace {

long long used_bytes(const mcv_server *s) {
  long long b = 0;
  for (const Pool *p : s->pools) b += p->bytes;
  return b;
}

long long footprint(const mcv_server *s, int order, int nc, int members) {
  return mcv_footprint_bytes(order, nc, s->scheme, s->precision, members);
}

int slots_for(const mcv_server *s, int order, int nc) {
  const long long per = footprint(s, order, nc, 2) - footprint(s, order, nc, 1);
  const long long n = s->slot_bytes / std::max(per, 1LL);
  return (int)std::max(1LL, std::min((long long)s->max_slots, n));
}

// Forget the cached groups that hold handle h (before its pool closes).
void drop_groups_of(mcv_server *s, const mcv_handle *h) {
  for (auto it = s->groups.begin(); it != s->groups.end();) {
    if (std::find(it->first.begin(), it->first.end(), h) != it->first.end()) {
      mcv_group_destroy(it->second);
      it = s->groups.erase(it);
    } else {
      ++it;
    }
  }
}

void close_pool(Pool *p) {
  if (p->h) {
    mcv_sync(p->h);
    mcv_destroy(p->h);
  }
  delete p;
}

// A pool on the grid (order, nc, dt), or nullptr with *rc = MCV_OK when the
// budget has no room for even one slot after evicting idle empty pools.  The
// pool gets slots_for() slots, fewer where the budget left by the pools that
// cannot be evicted (running, or holding a request) does not hold them: a
// request waits only while those pools leave no room for one slot, never for
// a pool larger than the budget (submit checked that one slot fits in it).
Pool *new_pool(mcv_server *s, int order, int nc, double dt, int *rc) {
  *rc = MCV_OK;
  long long pinned = 0;  // bytes of the pools that stay
  for (const Pool *q : s->pools)
    if (q->in_flight || !q->empty()) pinned += q->bytes;
  int slots = slots_for(s, order, nc);
  while (slots > 1 && pinned + footprint(s, order, nc, slots) > s->budget) --slots;
  const long long need = footprint(s, order, nc, slots);
  if (pinned + need > s->budget) return nullptr;
  while (used_bytes(s) + need > s->budget) {
    // evict an idle, empty pool (the largest first)
    Pool *victim = nullptr;
    for (Pool *p : s->pools)
      if (!p->in_flight && p->empty() && (!victim || p->bytes > victim->bytes)) victim = p;
    if (!victim) return nullptr;
    s->pools.erase(std::find(s->pools.begin(), s->pools.end(), victim));
    drop_groups_of(s, victim->h);
    close_pool(victim);
    ++s->pools_evicted;
  }
  Pool *p = new Pool();
  p->order = order;
  p->nc = nc;
  p->dt = dt;
  p->slots = slots;
  p->bytes = need;
  p->req.assign(slots, -1);
  p->left.assign(slots, 0);
  p->total.assign(slots, 0);
  if ((*rc = mcv_create(order, nc, s->scheme, s->precision, dt, s->radius, slots, &p->h)) != MCV_OK ||
      (*rc = mcv_set_geometry_equiangular(p->h)) != MCV_OK ||
      (s->tile >= 0 && (*rc = mcv_select_tile(p->h, s->tile)) != MCV_OK)) {
    close_pool(p);
    return nullptr;
  }
  s->pools.push_back(p);
  ++s->pools_created;
  return p;
}

int load_member(Pool *p, int slot, const Request &r) {
  if (r.spec)
    return mcv_set_member_balanced_flow(p->h, slot, r.gh0, r.u0, r.alpha, r.lmax, r.coef.empty() ? nullptr : r.coef.data(),
                                        r.rms, r.mh0, r.lon_c, r.lat_c, r.efold);
  return mcv_set_member(p->h, slot, r.phis.data(), r.u.data(), r.v.data(), r.phi.data());
}

int place(Pool *p, int slot, const Request &r) {
  if (int rc = load_member(p, slot, r)) return rc;
  p->req[slot] = r.id;
  p->left[slot] = r.nsteps;
  p->total[slot] = r.nsteps;
  p->active.push_back(slot);
  return MCV_OK;
}

// Admit r if a slot is free now: *placed = 1.  A request waits while the idle
// pools of its grid are full, a busy pool of its grid has a free slot (it is
// taken when that pool's chunk ends), or the budget has no room.
int admit(mcv_server *s, const Request &r, int *placed) {
  *placed = 0;
  bool busy_room = false;
  for (Pool *p : s->pools) {
    if (!p->same_grid(r.order, r.nc, r.dt)) continue;
    const int slot = p->free_slot();
    if (slot < 0) continue;
    if (p->in_flight) {
      busy_room = true;
      continue;
    }
    if (int rc = place(p, slot, r)) return rc;
    *placed = 1;
    return MCV_OK;
  }
  if (busy_room) return MCV_OK;
  int rc;
  Pool *p = new_pool(s, r.order, r.nc, r.dt, &rc);
  if (!p) return rc;
  if ((rc = place(p, 0, r))) return rc;
  *placed = 1;
  return MCV_OK;
}

// A pool's GPU time per step before its first chunk: ~1.3e-7 ms per point
// and step for one member (B200); the grouping policy compares pools with it.
double static_step_ms(const Pool *p) {
  const double n = 6. * std::pow((double)p->nc * (p->order - 1) + 1., 2.);
  return std::max(1.3e-7 * n * (double)p->active.size(), 0.02);
}

double step_ms(const Pool *p) { return p->ms_per_step > 0. ? p->ms_per_step : static_step_ms(p); }

// Grouping class of a pool: its order and its step cost's bucket on a
// log scale of base group_ratio (pools of one class step in lockstep).
long long group_class(const mcv_server *s, const Pool *p) {
  const double points = 6. * std::pow((double)p->nc * (p->order - 1) + 1., 2.);  // per member
  const long long b = (long long)std::floor(std::log(points) / std::log(std::max(s->group_ratio, 1.0001)));
  return (long long)p->order * 1000000 + b;
}

long long steps_left(const Pool *p) {
  long long left = p->left[p->active[0]];
  for (int slot : p->active) left = std::min(left, p->left[slot]);
  return left;
}

long long chunk_steps(const mcv_server *s, const Pool *p) {
  return std::max(1LL, std::min(steps_left(p), (long long)(s->chunk_ms / step_ms(p))));
}

// Record request `id` as failed with status rc (its result call reports rc).
void fail_request(mcv_server *s, long long id, long long nsteps, int rc) {
  Finished f;
  f.nsteps = nsteps;
  f.finite = 0;
  f.status = rc;
  s->finished[id] = std::move(f);
  s->unreported.push_back(id);
}

// The pool's chunk has ended: retire the forecasts it completed.  The step
// accounting and the slot lists are brought up to date before any call that
// can fail; a forecast whose check or read-back fails is retired as failed
// (its result call returns the error), so one bad forecast cannot wedge the
// loop.  Returns the first error seen.
int finish_chunk(mcv_server *s, Pool *p) {
  const long long steps = p->in_flight;
  p->in_flight = 0;
  p->group = nullptr;
  ++s->chunks;
  const double el = (now_ms() - p->launched) / (double)steps;
  p->ms_per_step = p->ms_per_step < 0. ? el : 0.5 * (p->ms_per_step + el);
  std::vector<int> done, still;
  for (int slot : p->active) {
    p->left[slot] -= steps;
    (p->left[slot] <= 0 ? done : still).push_back(slot);
  }
  p->active = still;
  if (done.empty()) return MCV_OK;
  std::vector<int> flags(p->slots, 0);
  int first = mcv_check_finite(p->h, flags.data());
  if (first == MCV_ERR_NONFINITE) first = MCV_OK;  // flagged per forecast below
  int npx, n, halo;
  mcv_grid_sizes(p->order, p->nc, &npx, &n, &halo);
  const size_t sz = (size_t)npx * npx * 6;
  for (int slot : done) {
    const long long id = p->req[slot];
    p->req[slot] = -1;
    int rc = first;
    Finished f;
    if (!rc) {
      f.u.resize(sz);
      f.v.resize(sz);
      f.phi.resize(sz);
      f.phiG.resize(sz);
      rc = mcv_get_state(p->h, slot, f.u.data(), f.v.data(), f.phi.data(), f.phiG.data());
    }
    if (rc) {
      fail_request(s, id, p->total[slot], rc);
      if (!first) first = rc;
      continue;
    }
    f.nsteps = p->total[slot];
    f.finite = flags[slot] ? 0 : 1;
    s->finished[id] = std::move(f);
    s->unreported.push_back(id);
  }
  return first;
}

int check_grid(int order, int nc, double dt, long long nsteps) {
  if (order != 3 && order != 4) return fail(MCV_ERR_ARG, "order must be 3 (MCV3) or 4 (MCV4)");
  if (nc < 2 || nc > 4096) return fail(MCV_ERR_ARG, "nc out of range [2, 4096]");
  if (!(dt > 0.) || !std::isfinite(dt)) return fail(MCV_ERR_ARG, "dt must be positive and finite");
  if (nsteps < 1) return fail(MCV_ERR_ARG, "nsteps must be >= 1");
  return MCV_OK;
}

}  // namespace

extern "C" int mcv_server_create(int precision, int scheme, double radius, long long hbm_budget,
                                 long long slot_bytes, int max_slots, double chunk_ms, int tile, mcv_server **out) {
  if (!out) return fail(MCV_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (precision != MCV_FP64 && precision != MCV_MIXED)
    return fail(MCV_ERR_ARG, "precision must be MCV_FP64 or MCV_MIXED");
  if (scheme != MCV_RK3_TVD && scheme != MCV_RK4) return fail(MCV_ERR_ARG, "scheme must be MCV_RK3_TVD or MCV_RK4");
  if (!(radius > 0.) || !std::isfinite(radius)) return fail(MCV_ERR_ARG, "radius must be positive and finite");
  if (slot_bytes < 1 || max_slots < 1) return fail(MCV_ERR_ARG, "slot_bytes and max_slots must be >= 1");
  if (!(chunk_ms > 0.) || !std::isfinite(chunk_ms)) return fail(MCV_ERR_ARG, "chunk_ms must be positive");
  if (tile < -1) return fail(MCV_ERR_ARG, "tile must be -1 (autotune) or a candidate index");
  if (hbm_budget <= 0) {
    long long free_b = 0, total_b = 0;
    if (int rc = mcv_device_memory(&free_b, &total_b)) return rc;
    hbm_budget = (long long)(0.85 * (double)free_b);
  }
  mcv_server *s = new mcv_server();
  s->precision = precision;
  s->scheme = scheme;
  s->radius = radius;
  s->budget = hbm_budget;
  s->slot_bytes = slot_bytes;
  s->max_slots = max_slots;
  s->chunk_ms = chunk_ms;
  s->tile = tile;
  *out = s;
  return MCV_OK;
}

extern "C" int mcv_server_submit(mcv_server *s, int order, int nc, double dt, long long nsteps, const double *phi_s,
                                 const double *u, const double *v, const double *phi, long long *id) {
  if (!s || !id) return fail(MCV_ERR_ARG, "server or id is NULL");
  if (int rc = check_grid(order, nc, dt, nsteps)) return rc;
  if (!phi_s || !u || !v || !phi) return fail(MCV_ERR_ARG, "state array is NULL");
  if (footprint(s, order, nc, 1) > s->budget) return fail(MCV_ERR_NOMEM, "the request's grid exceeds the HBM budget");
  int npx, n, halo;
  mcv_grid_sizes(order, nc, &npx, &n, &halo);
  const size_t sz = (size_t)npx * npx * 6;
  Request r{};
  r.id = s->next_id++;
  r.order = order;
  r.nc = nc;
  r.dt = dt;
  r.nsteps = nsteps;
  r.spec = false;
  r.phis.assign(phi_s, phi_s + sz);
  r.u.assign(u, u + sz);
  r.v.assign(v, v + sz);
  r.phi.assign(phi, phi + sz);
  s->waiting.push_back(std::move(r));
  *id = s->next_id - 1;
  return MCV_OK;
}

extern "C" int mcv_server_submit_balanced_flow(mcv_server *s, int order, int nc, double dt, long long nsteps,
                                               double gh0, double u0, double alpha, int lmax, const double *coef,
                                               double rms, double mountain_h0, double lon_c, double lat_c,
                                               double efold, long long *id) {
  if (!s || !id) return fail(MCV_ERR_ARG, "server or id is NULL");
  if (int rc = check_grid(order, nc, dt, nsteps)) return rc;
  if (lmax < 0 || lmax > 200 || (lmax > 0 && !coef)) return fail(MCV_ERR_ARG, "bad harmonic arguments");
  if (mountain_h0 > 0. && !(efold > 0.)) return fail(MCV_ERR_ARG, "bad mountain arguments");
  if (footprint(s, order, nc, 1) > s->budget) return fail(MCV_ERR_NOMEM, "the request's grid exceeds the HBM budget");
  Request r{};
  r.id = s->next_id++;
  r.order = order;
  r.nc = nc;
  r.dt = dt;
  r.nsteps = nsteps;
  r.spec = true;
  r.gh0 = gh0;
  r.u0 = u0;
  r.alpha = alpha;
  r.lmax = lmax;
  if (lmax > 0) r.coef.assign(coef, coef + (size_t)(lmax + 1) * (lmax + 1));
  r.rms = rms;
  r.mh0 = mountain_h0;
  r.lon_c = lon_c;
  r.lat_c = lat_c;
  r.efold = efold;
  s->waiting.push_back(std::move(r));
  *id = s->next_id - 1;
  return MCV_OK;
}

extern "C" int mcv_server_prepare(mcv_server *s, int order, int nc, double dt) {
  if (!s) return fail(MCV_ERR_ARG, "server is NULL");
  if (int rc = check_grid(order, nc, dt, 1)) return rc;
  for (Pool *p : s->pools)
    if (p->same_grid(order, nc, dt)) return MCV_OK;
  int rc;
  Pool *p = new_pool(s, order, nc, dt, &rc);
  if (!p) return rc ? rc : fail(MCV_ERR_NOMEM, "the HBM budget has no room for the pool");
  // a resting ocean in slot 0, stepped once: autotuning and graph capture
  // happen here and not inside a request's latency
  const int zero = 0;
  if ((rc = mcv_set_member_balanced_flow(p->h, 0, 2.94e4, 0., 0., 0, nullptr, 0., 0., 0., 0., 0.)) ||
      (rc = mcv_set_active(p->h, 1, &zero)) || (rc = mcv_step(p->h, 1)) || (rc = mcv_set_active(p->h, 0, nullptr)))
    return rc;
  p->dev_active.clear();
  p->dev_active_set = true;
  return MCV_OK;
}

extern "C" int mcv_server_poll(mcv_server *s, long long *ids, int max_ids, int *n_ids) {
  if (!s || !n_ids || max_ids < 0 || (max_ids > 0 && !ids)) return fail(MCV_ERR_ARG, "bad poll arguments");
  *n_ids = 0;
  // 1. chunks that ended (a failed query or read-back retires the pool's
  // finished forecasts as failed; the poll goes on and reports the error)
  int chunk_err = MCV_OK;
  for (Pool *p : s->pools) {
    if (!p->in_flight) continue;
    const int q = p->group ? mcv_group_query(p->group) : mcv_query(p->h);
    if (q == MCV_BUSY) continue;
    const int rc = (q != MCV_OK) ? q : finish_chunk(s, p);
    if (q != MCV_OK) {
      // the chunk's work is lost: its forecasts fail and their slots free up
      p->in_flight = 0;
      p->group = nullptr;
      for (int slot : p->active) {
        fail_request(s, p->req[slot], p->total[slot], q);
        p->req[slot] = -1;
      }
      p->active.clear();
    }
    if (rc && !chunk_err) chunk_err = rc;
  }
  // 2. admission, first come first served among the requests that fit
  // (a request whose initial state cannot be loaded is retired as failed and
  // its error returned once; the others stay queued)
  int first = MCV_OK;
  for (auto it = s->waiting.begin(); it != s->waiting.end();) {
    int placed;
    if (int rc = admit(s, *it, &placed)) {
      fail_request(s, it->id, it->nsteps, rc);
      if (!first) first = rc;
      it = s->waiting.erase(it);
      continue;
    }
    it = placed ? s->waiting.erase(it) : std::next(it);
  }
  // 3. the next chunk of every idle pool with active slots: alone on its
  // own stream, or (grouping) together with the idle pools of its class
  // (order and step-cost bucket), in one batched launch per stage
  auto fail_pool = [&](Pool *p, int rc) {
    // the pool cannot step: its forecasts fail and their slots free up
    for (int slot : p->active) {
      fail_request(s, p->req[slot], p->total[slot], rc);
      p->req[slot] = -1;
    }
    p->active.clear();
    if (!first) first = rc;
  };
  std::vector<Pool *> ready;
  for (Pool *p : s->pools) {
    if (p->in_flight || p->active.empty()) continue;
    if (!p->dev_active_set || p->dev_active != p->active) {
      if (int rc = mcv_set_active(p->h, (int)p->active.size(), p->active.data())) {
        fail_pool(p, rc);
        continue;
      }
      p->dev_active = p->active;
      p->dev_active_set = true;
    }
    ready.push_back(p);
  }
  if (s->group_max > 1) {
    // a pool whose class has a chunk on the GPU waits for it (at most one
    // chunk), so that the class's pools start their chunks together
    std::vector<long long> busy;
    for (const Pool *q : s->pools)
      if (q->in_flight) busy.push_back(group_class(s, q));
    ready.erase(std::remove_if(ready.begin(), ready.end(),
                               [&](const Pool *p) {
                                 return std::find(busy.begin(), busy.end(), group_class(s, p)) != busy.end();
                               }),
                ready.end());
  }
  std::stable_sort(ready.begin(), ready.end(), [&](const Pool *a, const Pool *b) {
    return group_class(s, a) < group_class(s, b);
  });
  for (size_t i = 0; i < ready.size();) {
    size_t j = i + 1;
    if (s->group_max > 1)
      while (j < ready.size() && (int)(j - i) < s->group_max && group_class(s, ready[j]) == group_class(s, ready[i]))
        ++j;
    mcv_group *grp = nullptr;
    if (j - i > 1) {
      std::vector<mcv_handle *> hs;
      for (size_t k = i; k < j; ++k) hs.push_back(ready[k]->h);
      auto it = s->groups.find(hs);
      if (it != s->groups.end()) {
        grp = it->second;
      } else if (mcv_group_create(hs.data(), (int)hs.size(), s->tile, &grp) == MCV_OK) {
        s->groups[hs] = grp;
      } else {
        grp = nullptr;  // (e.g. a pool's candidate is not a persistent TMA form): each pool alone
      }
    }
    if (!grp) {
      for (size_t k = i; k < j; ++k) {
        Pool *p = ready[k];
        const long long steps = chunk_steps(s, p);
        p->launched = now_ms();
        if (int rc = mcv_step_async(p->h, (int)steps)) {
          fail_pool(p, rc);
          continue;
        }
        p->in_flight = steps;
      }
      i = j;
      continue;
    }
    // one chunk for the group: the fewest steps any of its forecasts has left,
    // within chunk_ms of the pools' summed step times
    long long steps = steps_left(ready[i]);
    double ms = 0.;
    for (size_t k = i; k < j; ++k) {
      steps = std::min(steps, steps_left(ready[k]));
      ms += step_ms(ready[k]);
    }
    steps = std::max(1LL, std::min(steps, (long long)(s->chunk_ms / ms)));
    const double t = now_ms();
    if (int rc = mcv_group_step_async(grp, (int)steps)) {
      for (size_t k = i; k < j; ++k) fail_pool(ready[k], rc);
      i = j;
      continue;
    }
    ++s->grouped_chunks;
    for (size_t k = i; k < j; ++k) {
      ready[k]->launched = t;
      ready[k]->in_flight = steps;
      ready[k]->group = grp;
    }
    i = j;
  }
  // 4. the forecasts finished (or failed) since the last poll
  while (*n_ids < max_ids && !s->unreported.empty()) {
    ids[(*n_ids)++] = s->unreported.front();
    s->unreported.pop_front();
  }
  return chunk_err ? chunk_err : first;
}

extern "C" int mcv_server_result(mcv_server *s, long long id, double *u, double *v, double *phi, double *phiG,
                                 long long *nsteps, int *finite) {
  if (!s) return fail(MCV_ERR_ARG, "server is NULL");
  auto it = s->finished.find(id);
  if (it == s->finished.end()) {
    if (id >= 1 && id < s->next_id) {
      bool queued = false;
      for (const Request &r : s->waiting) queued = queued || r.id == id;
      for (const Pool *p : s->pools)
        for (long long r : p->req) queued = queued || r == id;
      if (queued) return MCV_BUSY;
    }
    return fail(MCV_ERR_ARG, "no such request (unknown, or its result was already taken)");
  }
  const Finished &f = it->second;
  if (f.status != MCV_OK) {
    const int st = f.status;
    if (nsteps) *nsteps = f.nsteps;
    if (finite) *finite = 0;
    s->finished.erase(it);
    for (auto q = s->unreported.begin(); q != s->unreported.end(); ++q)
      if (*q == id) {
        s->unreported.erase(q);
        break;
      }
    return fail(st, "the forecast failed (its initial state, a step or its read-back returned this error)");
  }
  const size_t bytes = f.u.size() * sizeof(double);
  if (u) std::memcpy(u, f.u.data(), bytes);
  if (v) std::memcpy(v, f.v.data(), bytes);
  if (phi) std::memcpy(phi, f.phi.data(), bytes);
  if (phiG) std::memcpy(phiG, f.phiG.data(), bytes);
  if (nsteps) *nsteps = f.nsteps;
  if (finite) *finite = f.finite;
  s->finished.erase(it);
  for (auto q = s->unreported.begin(); q != s->unreported.end(); ++q)
    if (*q == id) {
      s->unreported.erase(q);
      break;
    }
  return MCV_OK;
}

extern "C" int mcv_server_stats(mcv_server *s, long long *stats) {
  if (!s || !stats) return fail(MCV_ERR_ARG, "server or stats is NULL");
  long long running = 0, busy = 0;
  for (const Pool *p : s->pools) {
    for (long long r : p->req) running += r >= 0;
    busy += p->in_flight > 0;
  }
  stats[0] = (long long)s->waiting.size();
  stats[1] = running;
  stats[2] = (long long)s->finished.size();
  stats[3] = (long long)s->pools.size();
  stats[4] = busy;
  stats[5] = used_bytes(s);
  stats[6] = s->pools_created;
  stats[7] = s->pools_evicted;
  stats[8] = s->chunks;
  return MCV_OK;
}

extern "C" int mcv_server_set_grouping(mcv_server *s, int max_grids, double max_cost_ratio,
                                       long long *grouped_chunks) {
  if (!s) return fail(MCV_ERR_ARG, "server is NULL");
  if (max_grids < 1 || max_grids > 4 || !(max_cost_ratio >= 1.))
    return fail(MCV_ERR_ARG, "max_grids must be 1..4 and max_cost_ratio >= 1");
  s->group_max = max_grids;
  s->group_ratio = max_cost_ratio;
  if (grouped_chunks) *grouped_chunks = s->grouped_chunks;
  return MCV_OK;
}

extern "C" int mcv_server_destroy(mcv_server *s) {
  if (!s) return MCV_OK;
  for (Pool *p : s->pools)
    if (p->h) mcv_sync(p->h);
  for (auto &kv : s->groups) mcv_group_destroy(kv.second);
  s->groups.clear();
  for (Pool *p : s->pools) close_pool(p);
  delete s;
  return MCV_OK;
}
