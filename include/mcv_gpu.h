/*
 * mcv_gpu.h -- C ABI of the B200 implementation of MCV_SW's explicit RK step.
 *
 * The reference has no FFI: its time loop calls the Fortran subroutines
 *   RK4(stat(new), stat(old))       src/time_scheme_mod.F90:13-44
 *   RK3_TVD(stat(new), stat(old))   src/time_scheme_mod.F90:46-69
 * from src/MCV_SW.F90:57-60, on module-global arrays.  This header is the
 * drop-in boundary for that loop: a Fortran driver binds it with
 * iso_c_binding (an interface module of bind(C) declarations mirroring the
 * prototypes below), Python binds it with ctypes.
 *
 * Conventions
 *  - Every function returns an int status: 0 = OK, < 0 = error;
 *    mcv_last_error() returns a message for the last failing call on the
 *    calling thread.
 *  - Host arrays are FP64 (or int32) in the reference's Fortran layout:
 *    column-major (i, j, panel) over the padded point range
 *    i, j = ips..ipe (npx = nPVx + 2*nPVHalo points per direction), 6 panels;
 *    2x2 matrices are (2, 2, i, j, panel).  The library copies host arrays;
 *    it never keeps a host pointer.
 *  - A handle owns one CUDA stream and all device memory of one grid
 *    (order, Nc) with `members` independent states.  A handle is not
 *    thread-safe; different handles are independent.
 *  - There is no CPU fallback: without a usable sm_100 GPU, mcv_create fails.
 */
#ifndef MCV_GPU_H
#define MCV_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mcv_handle mcv_handle;

/* integral_scheme (src/parameters_mod.F90:228-235) */
#define MCV_RK3_TVD 3
#define MCV_RK4 4
/* arithmetic of the step */
#define MCV_FP64 0  /* FP64 throughout (the plain form)                      */
#define MCV_MIXED 1 /* FP32 tendencies on phi - mean, FP64 state accumulation */

/* status codes */
#define MCV_OK 0
#define MCV_ERR_ARG (-1)       /* invalid argument or size                   */
#define MCV_ERR_CUDA (-2)      /* CUDA runtime error / no usable GPU         */
#define MCV_ERR_NOMEM (-3)     /* device allocation failed                   */
#define MCV_ERR_ORDER (-4)     /* call order (e.g. step before geometry)     */
#define MCV_ERR_NONFINITE (-5) /* a member's state became NaN/Inf            */
#define MCV_BUSY 1             /* mcv_query: queued work still running (not an error) */

/* Message of the last failing call on this thread ("" if none). */
const char *mcv_last_error(void);

/* ---------------------------------------------------------------------
 * Core stepping API: replaces the RK4 / RK3_TVD calls of the time loop.
 * ------------------------------------------------------------------- */

/* Allocate a handle for `members` states on one grid.
 * Replaces initParameters / initStat / initTend (src/parameters_mod.F90:134-239,
 * src/stat_mod.F90:25-45, src/tend_mod.F90:17-28).  nc = 90/dx (cells per
 * panel edge), order = DOF (3 = MCV3, 4 = MCV4, src/constants_mod.F90:4-10),
 * dt in seconds; radius only documents the geometry passed to
 * mcv_set_geometry (it is not used by the step itself). */
int mcv_create(int order, int nc, int scheme, int precision, double dt, double radius, int members,
               mcv_handle **out);

/* Upload the grid geometry computed by the caller's mesh setup
 * (src/mesh_mod.F90:57-214, src/ghost_mod.f90:21-79): sqrtG, matrixG,
 * matrixIG, matrixA, matrixIA, f over the padded range, and the ghost
 * interpolation weights ghost%iref / ghost%coef as (nPVx, nPVHalo) arrays. */
int mcv_set_geometry(mcv_handle *h, const double *sqrtG, const double *matrixG, const double *matrixIG,
                     const double *matrixA, const double *matrixIA, const double *f, const int *ghost_iref,
                     const double *ghost_coef);

/* The same geometry computed on the device for the handle's (order, nc) and
 * radius: the equiangular metric, the edge-strip matrices and the ghost
 * weights that mcv_build_geometry + mcv_set_geometry produce, with no host
 * arrays and no upload (new grids in a serving process).  Same formulas as
 * mcv_build_geometry (src/projection_mod.F90:8-322, src/mesh_mod.F90:132-163,
 * src/ghost_mod.f90:21-79); the device math library's tan/cos/atan2/pow
 * differ from the host's by a few ulp. */
int mcv_set_geometry_equiangular(mcv_handle *h);

/* Copy the handle's metric back (no reference counterpart; it lets a caller
 * check the geometry a handle holds, e.g. one built on the device): sqrtG,
 * G^11, G^12, G^22, f over the padded range (Fortran layout) and the ghost
 * weights iref, coef as (nPVx, nPVHalo); any output may be NULL. */
int mcv_get_geometry(mcv_handle *h, double *sqrtG, double *ig11, double *ig12, double *ig22, double *f,
                     int *ghost_iref, double *ghost_coef);

/* Upload member m's surface geopotential phi_s and its state: covariant u, v
 * and phi over the full padded range, halo included (the first stage of the
 * first step reads the caller's halo as src/time_scheme_mod.F90:27 does). */
int mcv_set_member(mcv_handle *h, int m, const double *phi_s, const double *u, const double *v, const double *phi);

/* Member m's initial state generated on the device (no host arrays): the
 * seeded balanced flow of the host init chain -- the tilted solid-body flow
 * (gh0, u0, alpha; mcv_ic_tilted_zonal, src/test_case_mod.F90:118-120),
 * plus g times the real spherical harmonics of degrees 1..lmax with the
 * (lmax+1)^2 coefficients coef (mcv_ic_add_harmonics' ordering) rescaled to
 * the area-weighted RMS height rms in metres (weightsOnPV x sqrtG quadrature),
 * plus, if mountain_h0 > 0, the Gaussian mountain of height mountain_h0 m and
 * e-folding distance efold m centred at (lon_c, lat_c) (mcv_ic_add_mountain),
 * with the winds converted to covariant components (mcv_sphere_to_cov).
 * Replaces mcv_set_member for this member; needs the geometry first.  The
 * device math library and the order of the sums differ from the host chain's
 * by a few ulp. */
int mcv_set_member_balanced_flow(mcv_handle *h, int m, double gh0, double u0, double alpha, int lmax,
                                 const double *coef, double rms, double mountain_h0, double lon_c, double lat_c,
                                 double efold);

/* Replace member m's state (u, v, phi over the padded range) and keep its
 * phi_s: the per-step input of a driver that owns the state on the host.
 * Split precision keeps the member's mean-depth reference (a constant offset
 * of E that drops out of every derivative). */
int mcv_set_state(mcv_handle *h, int m, const double *u, const double *v, const double *phi);

/* Advance every member by nsteps RK steps (the loop of src/MCV_SW.F90:57-77
 * without history output).  Blocks until the steps are done. */
int mcv_step(mcv_handle *h, int nsteps);

/* Queue nsteps on the handle's stream and return without waiting. */
int mcv_step_async(mcv_handle *h, int nsteps);
/* Wait for the work queued on the handle's stream. */
int mcv_sync(mcv_handle *h);
/* MCV_OK if all work queued on the handle has finished, MCV_BUSY if some is
 * still running; never waits. */
int mcv_query(mcv_handle *h);

/* The members mcv_step / mcv_step_async advance: `count` distinct indices in
 * `members` (default after mcv_create: all of them).  The others keep their
 * state and step count untouched; with count = 0 a step enqueues nothing.
 * A request loop uses this to retire finished forecasts and admit new ones
 * into free member slots of a running handle.  No counterpart in the
 * reference (one state per run). */
int mcv_set_active(mcv_handle *h, int count, const int *members);

/* Failure detection (no counterpart in the reference, which writes NaNs to
 * its history files): waits for queued work, then flags[m] = 1 (host array of
 * `members`, may be NULL) where member m's interior u, v or phi holds a NaN or
 * Inf, else 0.  Returns MCV_ERR_NONFINITE if an active member is flagged. */
int mcv_check_finite(mcv_handle *h, int *flags);

/* Failure-path check, with no GPU fault, of the bounded wait the stage kernels
 * use on their staged copies (no reference counterpart): one warp waits on a
 * fresh mbarrier that nothing completes (complete = 0) or that is completed
 * first (complete = 1), giving up after limit_ms (0 < limit_ms <= 2000).
 * *timed_out = 1 if the wait gave up; *elapsed_ms = the wait's device time.
 * The stage kernels wait with a limit of about one second, then raise the flag
 * mcv_sync reports and return. */
int mcv_selftest_wait(int complete, double limit_ms, int *timed_out, double *elapsed_ms);

/* ---------------------------------------------------------------------
 * Groups: several grids in one persistent launch.  No counterpart in the
 * reference (one grid per process).  A group advances 1..4 handles of one
 * order, precision, scheme and device -- any Nc, dt and member counts -- with
 * one launch of the stage kernel per RK stage over the work items of all of
 * them (each grid with its own geometry, dt and state buffers), followed by
 * each grid's halo kernel; a group step is one CUDA graph.  tile: the
 * stage-kernel candidate of the launch (mcv_tuning's index of a persistent
 * TMA form), or -1 for the first handle's choice.  Each handle's result is
 * bit for bit that of the handle stepped alone on the same candidate.  The
 * handles keep working alone as well: the group orders its work after what
 * is queued on their streams, and their later work after the group's.
 * Destroy a group before any of its handles.
 * ------------------------------------------------------------------- */
typedef struct mcv_group mcv_group;
int mcv_group_create(mcv_handle *const *handles, int count, int tile, mcv_group **out);
/* Queue nsteps RK steps of every handle's active members (handles with none
 * are skipped); mcv_group_step also waits. */
int mcv_group_step_async(mcv_group *g, int nsteps);
int mcv_group_step(mcv_group *g, int nsteps);
/* Wait for the group's queued steps; reports a stage kernel's error flag. */
int mcv_group_sync(mcv_group *g);
/* MCV_OK if the group's queued steps have finished, MCV_BUSY otherwise. */
int mcv_group_query(mcv_group *g);
/* Advance nsteps and return their device time (CUDA events on the group's stream). */
int mcv_group_time_steps(mcv_group *g, int nsteps, double *ms);
int mcv_group_destroy(mcv_group *g);

/* Download member m's state over the padded range (any pointer may be NULL).
 * phiG = phi * sqrtG as src/time_scheme_mod.F90:85 stores it. */
int mcv_get_state(mcv_handle *h, int m, double *u, double *v, double *phi, double *phiG);

/* Total mass and energy of member m, with the quadrature of
 * calc_total_mass / calc_total_energy (src/diag_mod.F90:10-67), summed on the
 * device in FP64 with compensated (Neumaier) summation. */
int mcv_mass_energy(mcv_handle *h, int m, double *mass, double *energy);

/* History-output staging: the sequence the reference's time loop runs at a
 * history interval (src/MCV_SW.F90:62-67) on member m's device state, with
 * only the requested outputs crossing PCIe (any pointer may be NULL):
 *  - u, v, phi over the padded range with FillValue in the halo corner
 *    squares of u and v (addFillValue, src/output_mod.F90:230-248) and of phi
 *    once a step has run (src/ghost_mod.f90:161,179);
 *  - zonal, merid: convert_wind_P2SP over the whole padded range
 *    (src/spatial_operators_mod.F90:391-405) of those u, v, with A IG
 *    evaluated per point on the device from the equiangular formulas at the
 *    handle's radius (which must be the geometry's);
 *  - uC, vC, phiC: calc_VIA (src/diag_mod.F90:69-93) of u, v, phi with the
 *    reference's weightsOnPV (MCV4's /80 included, src/mesh_mod.F90:183-203),
 *    in stat%uC's layout (ics:ice, jcs:jce, 6) = (nc+2, nc+2, 6), halo cells 0.
 * A Fortran driver passes stat(new)'s arrays and calls history_write_stat
 * unchanged; calc_total_mass / calc_total_energy are mcv_mass_energy. */
int mcv_get_history(mcv_handle *h, int m, double *u, double *v, double *phi, double *zonal, double *merid,
                    double *uC, double *vC, double *phiC);

/* Normalized L1, L2 and Linf errors of doc/orderCheck.m:63-81 between the
 * calc_VIA cell averages of phi of member ma of handle a and member mb of
 * handle b (the reference), weighted by areaCell, computed on the device:
 * norms[0..2] = L1, L2, Linf.  Both handles hold the same grid on the same
 * device; b's queued work is waited for.  No reference counterpart (the
 * reference computes these offline in MATLAB from its history files). */
int mcv_height_error_norms(mcv_handle *a, int ma, mcv_handle *b, int mb, double *norms);

/* mesh%areaCell (src/mesh_mod.F90:205-212, EquiangularAllAreas :240-276):
 * cell areas in (ics:ice, jcs:jce, 6) = (nc+2, nc+2, 6) layout, halo cells 0.
 * Host only. */
int mcv_cell_areas(int nc, double radius, double *areaCell);

/* Instrumentation (no counterpart in the reference, which only prints its
 * total wall time, src/MCV_SW.F90:80-82).
 * mcv_time_steps: advance nsteps and return their device time (CUDA events on
 * the handle's stream around the replayed step graphs).
 * mcv_profile_step: advance nsteps launching every kernel directly with events
 * around each; returns the mean device time per launch of each stage kernel
 * (stage_ms[0..3], unused stages 0) and of the halo kernel. */
int mcv_time_steps(mcv_handle *h, int nsteps, double *ms);
int mcv_profile_step(mcv_handle *h, int nsteps, double *stage_ms, double *halo_ms);

/* Stage-kernel tile shapes the autotuner timed on this handle's grid (it runs
 * once, before the first step): ncand (at most 16) candidates,
 * shapes[6*i..] = {cells in x, cells in y, threads, sweep style (0 per-cell
 * items, n walks of n cells), CTAs per SM the kernel's registers allow, form
 * (0 one CTA per tile, 1 persistent CTAs with TMA-staged tiles)}, ms[i] =
 * device time per launch, *chosen = the index in use.  No counterpart in the
 * reference (which has no GPU path). */
int mcv_tuning(mcv_handle *h, int *ncand, int *chosen, int *shapes, float *ms);

/* Use candidate `index` of mcv_tuning's list instead of the autotuner's choice
 * (-1 re-runs the autotuner before the next step).  A shape is deterministic.
 * In FP64, shapes differ only in how the compiler contracts a*b+c into FMA
 * (last-bit differences); in split precision each tile also subtracts its own
 * linear reference before rounding to FP32, so shapes agree to FP32 rounding
 * of the residuals.  Pin one shape where results must match bit for bit. */
int mcv_select_tile(mcv_handle *h, int index);

/* Total mass and energy of `members` states that already live in the caller's
 * device memory, without allocating anything.  No counterpart in the reference
 * (its diagnostics, src/diag_mod.F90:10-67, run on host arrays); this is for
 * callers that cannot let a library allocate device memory when they ask for
 * diagnostics: code whose device memory is owned by a framework's caching
 * allocator, loops that must not pay for cudaMalloc/cudaFree, processes near
 * their memory budget.
 * Inputs are device pointers in the reference's layout: u, v, phi, phi_s as
 * (npx, npx, 6, members) and sqrtG as (npx, npx, 6), column-major, halo
 * included; matrixIG as (2, 2, npx, npx, 6).  mass, energy are host arrays of
 * `members`.  stream is a cudaStream_t (NULL: the default stream); the call
 * waits for its own work.  Limits: members <= 64.  The scratch (one partial sum
 * per block and member) is a fixed static device array of about 300 KiB held by
 * every device that loads the library; the first call on a device looks up its
 * address, so make that first call before any stream capture.  The address is
 * kept per device and context: after a device reset (a new primary context)
 * the next call looks it up again.  Calls that overlap on the GPU share the
 * scratch and race. */
int mcv_mass_energy_noalloc(int order, int nc, int members, const double *u, const double *v, const double *phi,
                            const double *phi_s, const double *sqrtG, const double *matrixIG, void *stream,
                            double *mass, double *energy);

/* Release the handle and its device memory. */
int mcv_destroy(mcv_handle *h);

/* Sizes of the grid: npx (padded points per direction), n (= nPVx), halo. */
int mcv_grid_sizes(int order, int nc, int *npx, int *n, int *halo);

/* Device bytes a handle with these arguments allocates (admission control). */
long long mcv_footprint_bytes(int order, int nc, int scheme, int precision, int members);

/* Free and total bytes of the current device (cudaMemGetInfo), for admission
 * control by HBM footprint. */
int mcv_device_memory(long long *free_bytes, long long *total_bytes);

/* ---------------------------------------------------------------------
 * Forecast server: continuous batching of many forecasts on one GPU.
 * No counterpart in the reference, which runs one forecast per process
 * (src/MCV_SW.F90).  Requests of any order, Nc, dt and length are queued;
 * each is admitted, by HBM footprint, into a free member slot of a pool (a
 * handle of its grid (order, Nc, dt) with device geometry, built by
 * mcv_set_geometry_equiangular), and advanced with the pool's other members
 * in chunks of RK steps on the pool's own stream, so pools of different grids
 * overlap on the GPU.  A request's result is bit for bit the one a plain
 * handle with the same tile shape gives it alone.  A server is not
 * thread-safe.
 * ------------------------------------------------------------------- */
typedef struct mcv_server mcv_server;

/* precision, scheme, radius: as mcv_create, for every pool.  hbm_budget:
 * bytes the pools may hold (<= 0: 85% of the device's free memory now).  A
 * pool gets as many slots as fit in slot_bytes (1..max_slots), fewer when the
 * budget left by the pools in use holds fewer.  chunk_ms: GPU
 * time of one chunk, which bounds how long a request waits for a busy pool of
 * its grid.  tile: stage-kernel candidate of every pool (mcv_select_tile), or
 * -1 for each pool's autotuner. */
int mcv_server_create(int precision, int scheme, double radius, long long hbm_budget, long long slot_bytes,
                      int max_slots, double chunk_ms, int tile, mcv_server **out);

/* Queue a forecast of nsteps RK steps of dt seconds from the host state
 * (phi_s, u, v, phi over the padded range, as mcv_set_member; copied).
 * *id identifies it (ids count up from 1).  MCV_ERR_NOMEM if even a
 * one-slot pool of its grid exceeds the budget. */
int mcv_server_submit(mcv_server *s, int order, int nc, double dt, long long nsteps, const double *phi_s,
                      const double *u, const double *v, const double *phi, long long *id);

/* Queue a forecast whose initial state is generated on the device at
 * admission (the arguments of mcv_set_member_balanced_flow). */
int mcv_server_submit_balanced_flow(mcv_server *s, int order, int nc, double dt, long long nsteps, double gh0,
                                    double u0, double alpha, int lmax, const double *coef, double rms,
                                    double mountain_h0, double lon_c, double lat_c, double efold, long long *id);

/* Create the pool of a grid ahead of its requests and step a resting state
 * once, so that autotuning and graph capture are not part of a request's
 * latency.  Blocks. */
int mcv_server_prepare(mcv_server *s, int order, int nc, double dt);

/* One pass of the request loop; never waits for the GPU.  Retires the chunks
 * that have ended (checking finished forecasts for NaN/Inf and downloading
 * them), admits waiting requests that fit, first come first served, and
 * queues the next chunk of every idle pool.  Writes up to max_ids ids of
 * forecasts finished since the last poll to ids (*n_ids of them); the rest
 * are reported by later polls.  A pool's first chunk autotunes its stage
 * kernel and captures its step graphs, which blocks (see mcv_server_prepare).
 * A forecast whose initial state, step or read-back fails is retired as
 * failed and reported with the finished ids (its mcv_server_result returns the
 * error); the poll returns the first such error and the loop goes on. */
int mcv_server_poll(mcv_server *s, long long *ids, int max_ids, int *n_ids);

/* Copy out and release a finished forecast: u, v, phi, phiG over the padded
 * range (any pointer may be NULL), its step count and *finite = 0 if its
 * state holds a NaN or Inf.  MCV_BUSY if it is still queued or running; the
 * forecast's error (and release) if it failed. */
int mcv_server_result(mcv_server *s, long long id, double *u, double *v, double *phi, double *phiG,
                      long long *nsteps, int *finite);

/* stats[9]: waiting requests, running forecasts, finished results not yet
 * taken, pools, pools with a chunk on the GPU, bytes the pools hold, pools
 * created, pools evicted, chunks retired. */
int mcv_server_stats(mcv_server *s, long long *stats);

/* Grouping: pools of one order whose grids' step costs (points per member)
 * fall in one bucket of a log scale of base max_cost_ratio form a class; a
 * class's idle pools advance together, up to max_grids (1..4) pools per
 * batched launch (mcv_group_*), and a pool whose class has a chunk on the GPU
 * waits for it (at most one chunk) so that the class starts together.
 * max_grids = 1 (the default): every pool on its own stream.  A grouped chunk
 * takes the fewest steps any of its forecasts has left.  Pools whose
 * stage-kernel candidate is not a persistent TMA form step alone.
 * *grouped_chunks (may be NULL): grouped chunks launched so far. */
int mcv_server_set_grouping(mcv_server *s, int max_grids, double max_cost_ratio, long long *grouped_chunks);

/* Release every pool and the server (waits for queued work). */
int mcv_server_destroy(mcv_server *s);

/* ---------------------------------------------------------------------
 * Host-side init chain (the caller's side of the boundary; provided so C,
 * C++ and Python callers without the Fortran setup can build inputs).
 * ------------------------------------------------------------------- */

/* Restates initMesh + initGhost (src/mesh_mod.F90:57-214,
 * src/projection_mod.F90:8-322, src/ghost_mod.f90:21-79): fills every padded
 * array; any output may be NULL. */
int mcv_build_geometry(int order, int nc, double radius, double *lonP, double *latP, double *sqrtG, double *matrixG,
                       double *matrixIG, double *matrixA, double *matrixIA, double *f, int *ghost_iref,
                       double *ghost_coef);

/* Williamson test cases 2, 5, 6 as initTestCase sets them
 * (src/test_case_mod.F90:52-191): sphere winds, phi and phi_s on the padded
 * points from lonP/latP. */
int mcv_ic_williamson(int case_num, long long npts, const double *lonP, const double *latP, double radius,
                      double *zonal, double *merid, double *phi, double *phi_s);

/* Balanced solid-body zonal flow with its axis tilted by alpha (the case-5
 * formulas of src/test_case_mod.F90:118-120 with no mountain). */
int mcv_ic_tilted_zonal(long long npts, const double *lonP, const double *latP, double radius, double gh0, double u0,
                        double alpha, double *zonal, double *merid, double *phi);

/* phi += scale * sum_{l=1..lmax, m=-l..l} c[l*l + l + m] * Y_lm(lon, lat),
 * with orthonormal real spherical harmonics (integral of Y^2 over the unit
 * sphere = 1). */
int mcv_ic_add_harmonics(long long npts, const double *lonP, const double *latP, int lmax, const double *coef,
                         double scale, double *phi);

/* Gaussian mountain hs = h0 * exp(-(d/efold)^2), d the great-circle distance
 * (m) to (lon_c, lat_c): phi_s = g*hs, phi -= g*hs (test_case_mod.F90:117-128). */
int mcv_ic_add_mountain(long long npts, const double *lonP, const double *latP, double radius, double lon_c,
                        double lat_c, double h0, double efold, double *phi, double *phi_s);

/* Adds one Rossby-Haurwitz wave of zonal wavenumber R (the case-6 formulas of
 * src/test_case_mod.F90:133-191 with wave number R and angular velocity omg,
 * without the constant gravity*h0) to zonal, merid and phi. */
int mcv_ic_add_rossby_haurwitz(long long npts, const double *lonP, const double *latP, double radius, int R,
                               double omg, double *zonal, double *merid, double *phi);

/* Adds one linear Rossby wave of zonal wavenumber R and amplitude K (1/s):
 * the wave part of the case-6 velocity (src/test_case_mod.F90:144-149)
 * without its solid-body rotation, and the cos(R lon) height term balancing
 * it at linear order (:160-164 with omega -> 0 in the factor Omega + omega). */
int mcv_ic_add_rossby_wave(long long npts, const double *lonP, const double *latP, double radius, int R, double K,
                           double *zonal, double *merid, double *phi);

/* Covariant winds from sphere winds, (u,v) = (G IA)(zonal, merid), as
 * initTestCase does (src/test_case_mod.F90:32-39, projection_mod.F90:60-77). */
int mcv_sphere_to_cov(long long npts, const double *matrixG, const double *matrixIA, const double *zonal,
                      const double *merid, double *u, double *v);

#ifdef __cplusplus
}
#endif

#endif /* MCV_GPU_H */
