/* SPDX-License-Identifier: Apache-2.0
 *
 * alloy_dfsph.h — C ABI of the B200 DFSPH liquid step (liballoy_dfsph.so).
 *
 * This is the drop-in boundary for the reference's SolverDFSPH (argonrobotics-ai/alloy, alloy/solvers/sph). Each entry
 * point names the reference interface it replaces. All particle arrays are in the caller's particle order (the
 * Newton model's), float32 vec3 as [n][3]; device pointers are CUDA device memory of the solver's device. Calls
 * return ADF_OK (0) or an ADF_ERR_* code; adf_last_error() gives the message of the calling thread's last failure.
 * No C++ exception or torch type crosses this boundary. adf_step allocates nothing.
 */
#ifndef ALLOY_DFSPH_H
#define ALLOY_DFSPH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADF_OK 0
#define ADF_ERR_VALUE 1    /* invalid argument or model layout (the reference raises ValueError) */
#define ADF_ERR_CAPACITY 2 /* a fixed capacity is exceeded (the reference raises CapacityError) */
#define ADF_ERR_CUDA 3     /* a CUDA runtime call failed */
#define ADF_ERR_STATE 4    /* the call is not valid in the solver's current state */

typedef struct adf_solver adf_solver;

/* Solver constants. Configuration fields follow DFSPHConfig (alloy/solvers/sph/config.py:46-131); the derived host
 * constants (sigma, n_full, tot_min, lattice_grad, wall_offset, wall_amplitude, taper0/1, reach, project_eps) are
 * the float64 values of config.py:225-236, kernels.py:221-270, layout.py:195-244 and solver.py:94, 483. */
typedef struct {
  int kind;                 /* 0 cubic spline, 1 Wendland C2 */
  double particle_radius;   /* r [m] */
  double h;                 /* support radius [m] */
  double sigma;             /* W(0) = 8/(pi h^3) or 21/(2 pi h^3) */
  double n_full;            /* neighbours of an interior lattice particle */
  double tot_min;           /* diagonal floor x lattice diagonal [1/m^2] */
  double lattice_grad;      /* sqrt(lattice diagonal) [1/m] */
  double wall_offset;       /* boundary fit delta [m] */
  double wall_amplitude;    /* boundary fit A */
  double taper0, taper1;    /* slot taper interval [m] */
  double reach;             /* slots kept below this phi [m] */
  double tol_den, tol_div;  /* max_density_error, max_divergence_error */
  double max_error_factor;
  int min_it, max_it;
  double omega;             /* jacobi_omega */
  double warm_den, warm_div;
  double min_nb;            /* min_neighbors_divergence */
  int divergence_solve, two_sided;
  double xsph_c;            /* 0: no XSPH */
  int capacity;             /* neighbor_capacity (8..64) */
  double v_sep;             /* contact_separation_speed [m/s] */
  double relief_speed;      /* compression_relief_speed [m/s]; <= 0: uncapped */
  double project_eps;       /* wall projection skin [m] */
  int has_bounds;           /* world_bounds given: escape box */
  double bounds_lo[3], bounds_hi[3];
  int cg;                   /* pressure iteration: 1 projected preconditioned CG per world (krylov.py:77-318; the
                               caller sets it only for one particle mass and rest density, solver.py:89-91),
                               0 relaxed Jacobi */
  int wall_friction;        /* Config.wall_friction: Coulomb friction of box walls on projected and lone particles */
  double skin;              /* [m] Verlet skin s = reneighbor_skin x h (neighbors_skin.py); 0: rows built every step.
                               Superset rows within h + s are reused per world until a particle of the world moves
                               more than s / 2 or the world's liquid set changes; the rows equal a plain build's */
  int skin_cap;             /* superset row capacity (neighbors_skin.py:155-166 skin_capacity) when skin > 0 */
  double jitter_speed;      /* [m/s] Config.rest_jitter_speed: the resting-jitter rule of the density solve's tolerance
                               (solve_driver.py:1-118); 0: off, every world stops at tol_den. On: per world and step
                               the tolerance is min(tol_den, v dt / H), floored at tol_den_min, with H the liquid's
                               hydrostatic depth from the density warm starts (1.5 sum k^2 / (|g| sum k)) and
                               v = max(jitter_speed, jitter_ratio |mean liquid velocity at the step's start|) */
  double jitter_ratio;      /* Config.rest_jitter_flow_ratio (0: v = jitter_speed) */
  double tol_den_min;       /* min(Config.min_density_error, max_density_error): the rule's floor */
} adf_params;

/* The model's particle arrays (Newton Model + sph:* attributes), bound once at creation. */
typedef struct {
  int n;                         /* particle count */
  int world_count;               /* W */
  const int32_t* world_start;    /* host [W + 1], contiguous worlds (Model.particle_world_start) */
  const float* q_host;           /* host [n][3] start positions: size the per-world grids (may be NULL) */
  const float* mass;             /* device [n] particle_mass */
  const float* rest_density;     /* device [n] sph:rest_density */
  const float* radius;           /* device [n] particle_radius (wall particles carry volume 8 r^3) */
  int32_t* flags;                /* device [n] particle_flags (written by emitters, sinks, the escape box) */
  int8_t* phase;                 /* device [n] sph:phase (written likewise) */
  const int32_t* world;          /* device [n] particle_world */
  const float* gravity;          /* device [W][3] Model.gravity */
  /* The liquid's static shape walls (layout.py:207-246 shape_table; boundary.py:70-87 per world: the world's own
   * shapes, then the global ones): boxes, spheres, capsules, straight cylinders and planes, each in its own frame.
   * n_shapes = 0: particle walls only, and the rest may be NULL. */
  int n_shapes;                  /* S: size of the model's shape table (ids index it; the particle wall's id is S) */
  const int32_t* shape_start;    /* host [W + 1]: world w's walls are shape_ids[shape_start[w] .. shape_start[w + 1]) */
  const int32_t* shape_ids;      /* host [shape_start[W]] */
  const float* shape_box;        /* host [S][8]: centre xyz, bounding radius, scale xyz (box half extents; sphere
                                    radius; capsule and cylinder radius, half height; plane width, length, 0 for an
                                    infinite plane), Coulomb friction */
  double sweep_len;              /* [m] a step longer than this is swept against the shapes: min(h, thinnest) / 2
                                    (integrate.py:42-49) */
  const int32_t* shape_geo;      /* host [S]: newton GeoType per shape (7 box, 3 sphere, 4 capsule and 6 cylinder along
                                    their z axis, 1 plane with normal z); NULL: all boxes */
  const float* shape_quat;       /* host [S][4]: the shape frame's rotation (x, y, z, w; unit); NULL: unrotated */
} adf_model;

/* Per-world host outputs of adf_get_report; any pointer may be NULL. SPHReport (types.py:11-28) and
 * WorldStats.diagnostics (runtime.py:410-418). Masses are int64 fixed point at 2^40 per kg. */
typedef struct {
  float* density_err;
  float* divergence_err;
  int32_t* iters_density;
  int32_t* iters_divergence;
  int64_t* mass_in;
  int64_t* mass_out;
  int64_t* mass_initial;
  int32_t* escaped;
  int32_t* neighbor_overflow;
  float* max_speed;
  float* density_err_max;
  int32_t* projected;
  int32_t* nonfinite;
  int32_t* emitter_overflow;
  float* density_tol;
  int32_t* learned_divergence; /* 1: the last step's divergence solve kept the learned start (adf_set_warm_model) */
  int32_t* learned_density;    /* the same for the density solve */
  int32_t* swept;              /* particles swept onto a box wall past a fast step (integrate.py:212-250), cumulative */
} adf_report;

/* Message of this thread's last failed call ("" if none). */
const char* adf_last_error(void);

/* Replaces SolverDFSPH.__init__ (solver.py:72-111): validates the layout (layout.py:47-72), binds the model arrays,
 * allocates every work array at fixed capacity and sizes the per-world cell grids. */
int adf_create(const adf_params* params, const adf_model* model, int device, adf_solver** out);

/* Frees the solver's device memory (the model's arrays are the caller's). */
void adf_destroy(adf_solver* solver);

/* Replaces SolverDFSPH.step (solver.py:218-268): one DFSPH step of every world. q_in/qd_in may alias q_out/qd_out;
 * f_ext (device [n][3] particle_f, N) may be NULL. Enqueued on `stream` (cudaStream_t; NULL: legacy default). */
int adf_step(adf_solver* solver, const float* q_in, const float* qd_in, float* q_out, float* qd_out,
             const float* f_ext, double dt, void* stream);

/* Step execution mode. enable = 1 (default): adf_step replays a CUDA graph of the whole step (built on first use per
 * state-pointer set and dt; the pressure iterations are WHILE nodes, as wp.capture_while, solve_driver.py:186);
 * 0: the same kernels launched one by one with the iteration count read back on the host. A step enqueued on a
 * stream that the caller is capturing always joins that capture with WHILE nodes. */
int adf_set_graphs(adf_solver* solver, int enable);

/* Autotuner (no counterpart in the reference; Warp picks its own launch shapes). enable = 1 (the default at creation):
 * the next adf_step on a stream that is not capturing is a tuning step: it launches its kernels one by one and, the
 * first time each neighbour-loop kernel (density and factor, solve start, pressure acceleration and its application,
 * Jacobi update, XSPH, list build) runs, times every candidate (threads per block {128, 256} x neighbour gathers in
 * flight {4, 8, 16}; for the list build 32 or 16 particles per warp) three times on that step's inputs and keeps the
 * fastest; it synchronises the stream while it does and
 * its results equal an ordinary step's bit for bit. 0: the default configuration (256 threads, 8 gathers). */
#define ADF_TUNE_KERNELS 6 /* density and factor, solve start, acceleration (and apply), Jacobi, XSPH, list build */
int adf_set_autotune(adf_solver* solver, int enable);
/* Pin one kernel's configuration (one of the tuner's candidates; for the list build block 128 and nb = particles per
 * warp, 32 or 16); the tuner then leaves it as set. */
int adf_set_tuned_config(adf_solver* solver, int kernel, int block, int nb);
/* The configuration in use per tuned kernel (host [ADF_TUNE_KERNELS] each, any may be NULL): threads per block,
 * gathers in flight, and the winning trial's milliseconds (-1 if not tuned). */
int adf_tuned_configs(adf_solver* solver, int32_t* block, int32_t* nb, float* ms);

/* Item halos of the Jacobi iterations (no reference counterpart; the reference gathers every neighbour from global
 * memory, pressure.py:264-352). The pressure acceleration and the Jacobi update run one block per 256-particle work
 * item; with halos, a kernel after the density pass lists per item the distinct particles its neighbour rows address
 * (at most 1,280) and rewrites the rows as 16-bit indices into that list, and the two kernels copy each item's records
 * into shared memory and gather from there. Items whose rows address more particles, or too wide a range of sorted
 * positions, keep the global gathers. Results are the same bits either way. mode 0 (the default at creation): global
 * gathers; 1: halos; -1: the autotuner times both forms with the other choices (its trials leave out the halo build,
 * which runs once per step). On a B200 the halos measured slower: the global gathers already hit L1 for about three
 * in four sectors, while the staged kernels' copy-in misses L1 and their shared memory halves the resident warps
 * (1M-particle dam break: 2.73 against 2.45 ms per step; the 4,096-world pour: 63.4 against 55.4 ms). The first
 * call with a nonzero mode allocates the halo buffers (6 bytes per row entry of the particle capacity, 5 KB per item)
 * and returns ADF_ERR_CAPACITY, leaving the mode unchanged, if the device has no room for them. */
int adf_set_halo(adf_solver* solver, int mode);

/* The halo choice in use (host int32[2]: acceleration, Jacobi; 1 = staged) and, after a step that built the halos,
 * host int64[4]: items staged, items left on global gathers, staged records summed over items, the largest item's
 * records. Synchronises `stream`. */
int adf_halo_stats(adf_solver* solver, int32_t* in_use, int64_t* stats, void* stream);

/* Persistent CG solve (no reference counterpart; the reference launches each CG kernel per iteration, krylov.py:254-297,
 * inside wp.capture_while, solve_driver.py:186). With the projected CG on models of at most 131,072 particles, each
 * pressure solve (its start and every iteration) runs as ONE cooperative launch whose phases are separated by
 * grid-wide barriers, instead of about nine launches per iteration; the results are the multi-launch path's bit for
 * bit. enable = 1 uses it wherever it applies (not in steps timed kernel by kernel, which take the multi-launch path);
 * 0 (the default at creation) takes the multi-launch path, which measured 2-4 % faster on a B200: under a replayed
 * step graph a grid barrier costs about what a kernel boundary does. Every barrier wait is bounded: a wait that gives
 * up sets the solver's status, after which adf_get_report returns ADF_ERR_STATE until adf_clear_status. */
int adf_set_persistent(adf_solver* solver, int enable);
/* Test hook of the bounded barrier waits: each wait polls at most `polls` times (default 4,194,304, about a second),
 * and a barrier waits for `extra_arrivals` more blocks than the grid has (default 0; any other value makes every wait
 * run out, which is what the wait-expiry test checks). */
int adf_set_barrier_wait(adf_solver* solver, long long polls, int extra_arrivals);
/* Clears the status words of the bounded waits (the persistent solve's barriers and the warm-start network's
 * tensor-core waits) and the per-world reduction tickets a launch that gave up may have left counted, after
 * synchronising the device. */
int adf_clear_status(adf_solver* solver);

/* Replaces SolverDFSPH.prime (solver.py:369-372, prime.py:52-87): with the divergence warm starts holding the
 * hydrostatic guess x dt (adf_set_warm_starts), one divergence solve of the velocity a gravity step adds to the
 * state (tolerance tol, up to max_it iterations, plain start 1 x the guess, no neighbour floor, no max-error test);
 * the state is not changed; afterwards the density warm start is kd = kv dt and kv = 0. iters (host, may be NULL)
 * receives the largest per-world iteration count; synchronises `stream` when iters is given. Not capturable. */
int adf_prime(adf_solver* solver, const float* q, const float* qd, double dt, double tol, int max_it, int32_t* iters,
              void* stream);

/* Replaces SolverDFSPH.density_ratio (solver.py:386-393): density ratio and active mask of every particle of the
 * state (device [n] outputs, 0 for non-liquid particles) from fresh lists and wall slots. */
int adf_density_ratio(adf_solver* solver, const float* q, const float* qd, float* ratio_out, float* active_out,
                      void* stream);

/* Replaces SolverDFSPH.report (solver.py:365-367) and stats.diagnostics: synchronises `stream`, copies to host. */
int adf_get_report(adf_solver* solver, adf_report* out, void* stream);

/* Replaces WorldStats._active_mass (runtime.py:381-385): int64 fixed-point liquid mass per world, host [W]. */
int adf_active_mass(adf_solver* solver, int64_t* out_host, void* stream);

/* Warm starts k dt (divergence) and k dt^2 (density) per particle: the alloy_state_arrays keys "sph.kappa_v" and
 * "sph.kappa_d" (coupling_hooks.py:260-271). Device [n] copies in particle order. */
int adf_get_warm_starts(adf_solver* solver, float* kappa_v, float* kappa_d, void* stream);
int adf_set_warm_starts(adf_solver* solver, const float* kappa_v, const float* kappa_d, void* stream);

/* The solver's own warm-start storage (device [n] float32 each, particle order), for snapshot code that saves and
 * restores "sph.kappa_v" / "sph.kappa_d" in place (coupling_hooks.py:260-271). Valid until adf_destroy. */
int adf_state_arrays(adf_solver* solver, float** kappa_v, float** kappa_d);

/* The rest of a snapshot's solver state, beside the warm starts: the keys that WorldStats.state_arrays
 * (runtime.py:173-174), EmitterManager.state_arrays (runtime.py:389-399) and SPHPort.state_arrays (ports.py:201-203)
 * add to alloy_state_arrays (coupling_hooks.py:115-138). Every pointer is the solver's own device storage, for
 * snapshot code that copies the arrays out and back in place between steps; the emitter pointers change when
 * emitters are added (adf_add_emitter(s)), all end with adf_destroy. */
typedef struct {
  int64_t* mass_in;       /* [W] "sph.mass_in": liquid mass emitted, int64 fixed point at 2^40 per kg */
  int64_t* mass_out;      /* [W] "sph.mass_out": liquid mass retired (sinks, escape box, port) */
  int32_t* escaped;       /* [W] "sph.escaped" */
  float* emit_t;          /* [E] "sph.emit_t": layer clocks [s]; NULL without emitters */
  int32_t* emit_cursor;   /* [E] "sph.emit_cursor": pool particles already emitted */
  int32_t* emit_world;    /* [E] each emitter's world: alloy_state_worlds' map of the two emitter keys */
  int32_t n_emitters;     /* E */
  int32_t* port_stack;    /* [n] "sph.port_stack": world w's held particles, a stack in its index range
                             [world_start[w], world_start[w + 1]) (the reference's [W][depth] stack, world by world) */
  int32_t* port_top;      /* [W] "sph.port_top": held particles per world */
  int32_t* port_absorbed; /* [W] "sph.port_absorbed" (cumulative since creation or reset) */
  int32_t* port_emitted;  /* [W] "sph.port_emitted" */
  int32_t* port_retired;  /* [W] "sph.port_retired" */
  int32_t* port_taken;    /* [W] the last absorb / retire call's count per world (SPHPort.taken) */
  int32_t* port_granted;  /* [W] the last port emit's count per world (SPHPort.granted) */
  int32_t n_patch_entries;  /* entries of all patch emitters (adf_add_patch_emitter), group after group */
  int32_t* patch_pending;   /* [entries] "sph.patch_pending{k}" (group k's slice) */
  int32_t* patch_fired;     /* [entries] "sph.patch_fired{k}" */
  int32_t* patch_world;     /* [entries] world of each entry (alloy_state_worlds) */
  int32_t* warm_probe_gap;  /* [2][W] with a warm-start network under the judge (NULL before adf_set_warm_model): solves
                               between evaluations of the learned start per solve kind (divergence, density) */
  int32_t* warm_probe_wait; /* [2][W] solves left before the next evaluation */
} adf_state_storage;
int adf_get_state_storage(adf_solver* solver, adf_state_storage* out);

/* Replaces SolverDFSPH.add_patch_emitter (solver.py:449-453, patch.py:146-187): a triggered one-shot emitter. One
 * entry per world e < entries: world[e], count[e] points (host float [sum count][3], world frame: this path has no
 * bodies) and as many spare particle ids (host int32 [sum count], reserved by the caller, patch.py:189-196), entry
 * after entry; velocity (host [3]) is the group's. Returns the group id (>= 0) or -ADF_ERR_*. Step graphs are
 * re-recorded on the next step. */
int adf_add_patch_emitter(adf_solver* solver, int entries, const int32_t* world, const int32_t* count,
                          const int32_t* pool_ids, const float* points, const float* velocity);

/* Replaces SolverDFSPH.trigger (solver.py:455-458, patch.py:199-210): arm group pid's entries whose world is set in
 * world_flags (device [W]; int32, or bool bytes when flags_bool = 1) and has not fired; at the end of the next step
 * each armed entry emits its particles once (liquid at its points with the group's velocity, mass into mass_in) and
 * fires. One launch, capture-safe. adf_reset re-arms the masked worlds' entries. */
int adf_trigger(adf_solver* solver, int pid, const void* world_flags, int flags_bool, void* stream);

/* Replaces SPHPort.absorb and SPHPort.retire (ports.py:101-122, 183-189; SolverDFSPH.retire, solver.py:428-431): the
 * masked liquid particles (mask: device int32 [n], non-zero = take) leave the liquid in one launch: ACTIVE cleared,
 * their velocity in qd (device [n][3], the state's) zeroed, their mass booked to mass_out. keep = 1 holds them for
 * adf_port_emit (phase -3, pushed on the world's stack in ascending id order), keep = 0 retires them for good (phase
 * -2). Counts go to port_taken and the cumulative port_absorbed / port_retired. Capture-safe; no host work. The port
 * books no flux energy (the reference's emitter energy export, emitters.flux_add, is not on this path). */
int adf_port_take(adf_solver* solver, float* qd, const int32_t* mask, int keep, void* stream);

/* Replaces SPHPort.emit (ports.py:191-199): per world the first min(n_req[w], R) requests (n_req: device int32 [W])
 * pop held particles (fewer when the world's reservoir runs out), which become liquid at pos [W][R][3] with velocity
 * vel [W][R][3] (device, world frame), written into q / qd (device [n][3], the state's), their mass booked into
 * mass_in; port_granted[w] says how many. Capture-safe. */
int adf_port_emit(adf_solver* solver, float* q, float* qd, const float* pos, const float* vel, int R,
                  const int32_t* n_req, void* stream);

/* Replaces SolverDFSPH.alloy_energy (solver.py:469-470; runtime.py:66-79, 423-430): kinetic plus gravity energy [J]
 * of each world's liquid about (0, 0, z_ref[w]) (z_ref: device float64 [W]) into out (device float64 [W]): per
 * particle m (v.v / 2 - g.(x - z_ref e_z)) in float64 from float32 dot products, summed in the per-world reductions'
 * fixed chunk and tree order. Allocates nothing; capture-safe. */
int adf_energy(adf_solver* solver, const float* q, const float* qd, const double* z_ref, double* out, void* stream);

/* Replaces SolverDFSPH.alloy_stable_dt (solver.py:465-467; runtime.py:55-62, 82-90, 411-421): out[w] (device float32
 * [W]) = dt_max for a world whose liquid is at rest, else clamp(cfl 2r / |v|max, dt_min, dt_max) over the state's
 * liquid (qd: device [n][3]; a non-finite speed counts as 1e30). Allocates nothing; capture-safe. */
int adf_stable_dt(adf_solver* solver, const float* qd, double cfl, double dt_min, double dt_max, float* out,
                  void* stream);

/* Replaces SolverDFSPH.reset (solver.py:353-362) + WorldStats.reset (runtime.py:431-449) + emitters.rewind
 * (emitters.py:241-255) + SPHPort.reset (ports.py:205-216): masked worlds (host [W] bytes; NULL = all) get warm
 * starts cleared, flags and phase back to flags0/phase0 (device [n]), their counters and ledgers zeroed, their
 * emitters rewound and their port reservoir back to its build-time particles. */
int adf_reset(adf_solver* solver, const uint8_t* world_mask, const int32_t* flags0, const int8_t* phase0,
              void* stream);

/* Replaces EmitterManager.add_emitter (runtime.py:498-525) after its host logic: a layer emitter with its layer
 * offsets (host [n_off][3], region frame), transform (px py pz qx qy qz qw), velocity, interval [s] and its pool of
 * spare particle ids (host, ascending). Returns the emitter index (>= 0) or -ADF_ERR_*. Between steps only. */
int adf_add_emitter(adf_solver* solver, int world, const float* xform, const float* offsets, int n_off,
                    const float* velocity, float interval, const int32_t* pool, int pool_size);

/* Many emitters in one call, with one upload of the emitter tables (adding them one by one re-uploads the tables each
 * time): emitter k has world[k], xform[k][7], n_off[k] offsets (the next n_off[k] rows of offsets[][3]), velocity[k][3],
 * interval[k] and pool_size[k] pool ids (the next pool_size[k] of pool). All are checked before any is added. Returns
 * the first new emitter's index (>= 0) or -ADF_ERR_*. Between steps only. */
int adf_add_emitters(adf_solver* solver, int count, const int32_t* world, const float* xform, const int32_t* n_off,
                     const float* offsets, const float* velocity, const float* interval, const int32_t* pool_size,
                     const int32_t* pool);

/* Replaces the pool reassignment of emitters.split_pools (emitters.py:225-238): emitter `emitter` draws from `pool`
 * (host ids, ascending) from now on; its cursor is kept. Between steps only. */
int adf_set_emitter_pool(adf_solver* solver, int emitter, const int32_t* pool, int pool_size);

/* Layer clocks [s] and cursors (particles of the pool already emitted) of every emitter, host arrays
 * (EmitterDevice.t_acc / cursor, emitters.py:174-213); either may be NULL. */
int adf_emitter_state(adf_solver* solver, float* t_acc, int32_t* cursor);

/* Replaces SolverDFSPH.set_emitter_enabled (solver.py:438-447). */
int adf_set_emitter_enabled(adf_solver* solver, int emitter, int enabled);

/* Replaces EmitterManager.add_sink (runtime.py:557-565): retire liquid entering the box (xform, half extents). */
int adf_add_sink(adf_solver* solver, int world, const float* xform, const float* half_extents);

/* Replaces NeighborLists.global_rows (neighbors.py:285-295): the last step's lists as global particle ids, host
 * rows [n][capacity] (entries past count are -1) and counts [n]; synchronises `stream`. */
int adf_neighbor_rows(adf_solver* solver, int32_t* rows, int32_t* count, void* stream);

/* Diagnostics for parity tests: a per-particle float field of the last step in particle order (device [n] or
 * [n][3]): ratio alpha neff reg src kappa lower err slot_psi slot_phi pred_kv pred_kd (scalars; pred_*: the
 * warm-start network's predictions), acc slot_g slot_vb slot_n (vec3). A slot field takes a ":k" suffix for slot k
 * (0..3 with box walls, nearest first; 0 without a suffix). slot_shape:k gives slot k's wall id (-1 empty; the particle
 * wall's id is n_shapes) and slot_count the slots in use, as floats, for liquid particles (0 elsewhere). */
int adf_debug_field(adf_solver* solver, const char* name, float* out, void* stream);

/* Replaces SkinState.rebuilt_worlds (neighbors_skin.py:206-208): host [W], 1 where the last step (or density_ratio)
 * rebuilt the world's superset rows; synchronises `stream`. ADF_ERR_STATE without a skin. */
int adf_skin_flags(adf_solver* solver, int32_t* flags, void* stream);

/* Per-world float64 sums and maxima of a float array in the solver's tree order (reduce.py:185-227); device
 * in/out; exported for the reducer's parity test. */
int adf_world_sum(adf_solver* solver, const float* values, double* out_sum, float* out_max, void* stream);

/* No counterpart in the reference. The per-world float64 sum and maximum of adf_world_sum, for callers that cannot
 * allocate device memory: a host loop that must not enter the CUDA allocator (cudaMalloc may synchronise the device
 * and has no latency bound), or a process whose device memory is already reserved by another framework's pool. It
 * needs no solver object and allocates nothing. values: device [n]; world_start: device [W + 1], non-decreasing,
 * world_start[W] <= n; out_sum: device [W] float64; out_max: device [W] float32, floored at 0. The result equals
 * adf_world_sum's for the same world ranges (same chunks, same tree order). Runs on the current device.
 * Scratch: a fixed static device array of about 0.85 MB, held by every GPU that loads the library until the process
 * exits. Limits: W <= ADF_NOALLOC_MAX_WORLDS and n / 256 + W + 1 <= ADF_NOALLOC_MAX_CHUNKS (about 12.5 million
 * values); larger sizes return ADF_ERR_CAPACITY with a message. The first call on a device sets up (looks up the
 * scratch's device address once, with that device current); make it before any stream capture. The address is kept
 * for the life of the process: it assumes the device's context does too (after a cudaDeviceReset or a torn-down
 * primary context it would be stale). All calls on a device share the scratch, so calls that overlap on the GPU (on
 * different streams) race. A world_start that decreases, or exceeds n, gives unspecified sums: every index is
 * clamped, so nothing is read or written outside the arrays, but chunks past the scratch's count are dropped. */
#define ADF_NOALLOC_MAX_WORLDS 16384
#define ADF_NOALLOC_MAX_CHUNKS 65536
int adf_world_sum_noalloc(const float* values, int n, const int32_t* world_start, int world_count, double* out_sum,
                          float* out_max, void* stream);

/* ------------------------------------------------------------------------------------------- warm-start network
 * No counterpart in the reference (its warm start is the previous step's kappa scaled, pressure.py:214-261). A per-
 * particle network 16 -> 64 -> 64 -> 2 (SiLU; BF16 weights, FP32 accumulation on the tcgen05 tensor cores) that predicts
 * both pressure solves' warm starts. Parameters are FP32 in one packed host vector of ADF_MLP_PARAMS floats:
 * W1[64][16], b1[64], W2[64][64], b2[64], W3[2][64], b3[2] (weights [out][in]). Feature rows are [n][16] FP32, target
 * rows [n][2] FP32, both normalised by the caller (adf_set_warm_model takes the statistics). */
#define ADF_MLP_PARAMS 5378
#define ADF_MLP_FEATURES 16
typedef struct adf_mlp adf_mlp;
int adf_mlp_create(const float* params, int device, adf_mlp** out);
void adf_mlp_destroy(adf_mlp* mlp);
/* Replace the parameters (host vector) and clear the Adam moments. */
int adf_mlp_set_params(adf_mlp* mlp, const float* params);
int adf_mlp_get_params(adf_mlp* mlp, float* params);
/* y[n][2] = network(x[n][16]) on the device (normalised units). */
int adf_mlp_forward(adf_mlp* mlp, const float* x, int n, float* y, void* stream);
/* Gradient (host [ADF_MLP_PARAMS], may be NULL) and loss (host [1], may be NULL) of L = sum (y - t)^2 / (2 batch) over
 * the rows idx[0 .. batch) (device int32) of x and targets t (device); synchronises `stream`. */
int adf_mlp_gradient(adf_mlp* mlp, const float* x, const float* t, const int32_t* idx, int batch, float* grad,
                     float* loss, void* stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) at learning rate lr on the same loss; loss (host, may be NULL: no
 * synchronisation) receives the batch's loss before the step. */
int adf_mlp_train_step(adf_mlp* mlp, const float* x, const float* t, const int32_t* idx, int batch, float lr,
                       float* loss, void* stream);
/* ADF_OK, or ADF_ERR_STATE if a tensor-core wait of this network's kernels ever expired (its results are invalid). */
int adf_mlp_status(adf_mlp* mlp);
/* Test hooks of the bounded waits. A tensor-core step's wait on its MMA's mbarrier gives up after `polls` polls
 * (default 2^22, far above a normal wait's few): the kernel then sets the status, waits (at most 2^22 polls) for the
 * MMAs it committed, frees its tensor memory and returns. polls = 0 makes every such wait give up at once, which runs
 * that path without any fault. adf_mlp_clear_status resets the status after a synchronisation. */
int adf_mlp_set_wait_limit(adf_mlp* mlp, uint32_t polls);
int adf_mlp_clear_status(adf_mlp* mlp);

/* Learned warm start (no counterpart in the reference; its starts are the previous kappa scaled, pressure.py:214-261).
 * With a network set, each step evaluates it once per liquid particle at the start of its first solve and both
 * solves begin from its predictions: the first Jacobi sweep runs from the plain and from the learned start, and a
 * world continues from the learned one unless its residual is larger (then the solve is exactly the plain one).
 * The network's weights are copied (the adf_mlp may be destroyed afterwards); norm is host [36]: feature mean[16],
 * 1 / feature deviation[16], target mean[2], target deviation[2]. model = NULL switches the learned start off.
 * Between steps only; the first call allocates the buffers of the learned start. */
int adf_set_warm_model(adf_solver* solver, const adf_mlp* model, const float* norm);
/* The network's two outputs are corrections, in the dt-free units of the stored warm starts (kappa dt and
 * kappa dt^2), to the plain starts 0.5 min(kappa_v, 0.5) and 0.9 min(kappa_d, 2.5e-4) (warm_div / warm_den); the
 * learned start is the plain start plus the correction, capped at 0.5 and 2.5e-4 and kept above the solve's lower
 * bound. */

/* First-sweep judging of the learned start (default 1, as described above). 0 measures the network alone: every world
 * starts from the learned kappa without the plain start's sweep; every world still iterates to the same tolerance. */
int adf_set_warm_judging(adf_solver* solver, int enable);

/* Record the network's 16 raw features of every liquid particle at the start of each step's first solve (always on
 * while a network is set); adf_warm_features copies the last step's record to out (device [n][16], particle order,
 * zero rows for other particles). Used to build training pairs with the converged warm starts (adf_get_warm_starts
 * after the step). */
int adf_set_feature_recording(adf_solver* solver, int enable);
int adf_warm_features(adf_solver* solver, float* out, void* stream);

/* Number of kernels this library enqueued since creation (launch accounting for benchmarks). */
int64_t adf_kernel_launches(const adf_solver* solver);

/* Live kernel timing with CUDA events on the launch stream (benchmarks). Kinds, in this order: 0 sort (classify,
 * scan, scatter), 1 neighbour rows, 2 wall slots, 3 density and factor, 4 solve start, 5 pressure acceleration,
 * 6 Jacobi update, 7 per-world reduction and stop test, 8 apply pressure, 9 XSPH, 10 advect/project/write-back,
 * 11 emitters, 12 warm-start network and learned start, 13 item halos. adf_profile_read synchronises, returns the summed
 * milliseconds and launch counts per kind since the last read (host arrays of ADF_PROF_KINDS) and starts a new
 * window. */
#define ADF_PROF_KINDS 14
int adf_profile_enable(adf_solver* solver, int enable);
int adf_profile_read(adf_solver* solver, double* ms, int64_t* launches);

/* Liquid particles covered by the Jacobi iterations' work lists since creation (each iteration's acceleration and
 * update kernels process the liquid of the worlds still iterating; benchmarks divide by launches for the particles
 * per launch). Host output; synchronises `stream`. */
int adf_iteration_work(adf_solver* solver, int64_t* particles, void* stream);

/* Liquid particle count and neighbour-row entries of the last list build (host outputs; synchronises `stream`). */
int adf_list_stats(adf_solver* solver, int32_t* fluid, int64_t* entries, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ALLOY_DFSPH_H */
