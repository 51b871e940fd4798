/*
 * mdpd.h -- C ABI of the B200 DPD/mDPD timestep library (libmdpd.so).
 *
 * Drop-in boundary for the USER-MESO hot path.  In the reference, LAMMPS core reaches
 * the path through its compile-time style registry and virtual methods:
 *   PairStyle(mdpd/meso, MesoPairMDPD)        src/USER-MESO/pair_mdpd_meso.h:3
 *   PairStyle(dpd/meso, MesoPairDPD)          src/USER-MESO/pair_dpd_meso.h:3
 *   AtomStyle(mdpd/atomic/meso, ...)          src/USER-MESO/atom_vec_mdpd_atomic_meso.h:3
 *   FixStyle(nve/meso / aboundary/rho/meso / aboundary/meso / addforce/meso / density/meso, ...)
 *   IntegrateStyle(mvv/meso, ModifiedVerlet)  src/USER-MESO/mvv_meso.h:3-4
 *   Input::file/one -> Force::create_pair / Modify::add_fix / Run::command (src/run.cpp:170-178)
 * A caller replaces that chain by these entry points.  Every call returns an MDPD_* status;
 * the library never exits the process (the reference aborts through error->all or
 * raise(SIGABRT), src/USER-MESO/util_meso.h:100-101, and exits on OOM, engine_meso.h:126-145).
 * All pointers are host pointers; the library owns every device allocation.
 */
#ifndef MDPD_H
#define MDPD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MDPD_OK 0
#define MDPD_ERR_PARSE 1     /* malformed or unsupported script command            */
#define MDPD_ERR_OOM 2       /* device allocation failed                            */
#define MDPD_ERR_OVERFLOW 3  /* neighbour list / ghost / bin capacity exceeded      */
#define MDPD_ERR_NAN 4       /* non-finite force                                    */
#define MDPD_ERR_TIMEOUT 5   /* bounded device wait expired                         */
#define MDPD_ERR_CUDA 6      /* CUDA runtime error                                  */
#define MDPD_ERR_ARG 7       /* invalid argument                                    */
#define MDPD_ERR_STATE 8     /* call out of order (e.g. run before the box exists)  */
#define MDPD_ERR_BUDGET 9    /* serving: job does not fit the HBM budget            */

typedef struct mdpd_s mdpd_t;

typedef struct mdpd_opts {
    int device;   /* CUDA device ordinal */
    int verbose;  /* echo the thermo log to stdout */
} mdpd_opts;

typedef struct mdpd_thermo_t {
    int64_t step;
    int64_t natoms;
    int64_t nbuild;       /* neighbour-list builds so far */
    double temp;          /* compute temp/meso over all atoms, dof = 3N-3 */
    double press;         /* compute pressure/meso scalar */
    double pe;            /* total pair energy (E_pair * N) */
    double ke;            /* 0.5 * sum m v^2 */
    double virial[6];     /* xx yy zz xy xz yz, sums of the per-atom halved virials */
    double momentum[3];
    double temp_group;    /* temperature of the nve/meso group */
    double ptensor[6];    /* pressure tensor (kinetic + virial)/V: xx yy zz xy xz yz */
    double surface_tension; /* (Lx/2)(Pxx - (Pyy+Pzz)/2) for a slab normal to x */
    int32_t status;       /* device error bits: 1 list, 2 ghost, 4 bin/bucket overflow, 8 non-finite
                             force, 16 particle lost, 32 compact list overflow, 64 index out of
                             range (index-check build) */
    int32_t pad;
} mdpd_thermo_t;

/* --- single box driven by the LAMMPS script surface ------------------------------------ */
/* Input::one / Input::file (src/input.cpp) for the supported command subset */
int mdpd_create(mdpd_t **h, const mdpd_opts *opts);
int mdpd_command(mdpd_t *h, const char *line);
int mdpd_file(mdpd_t *h, const char *path);
/* Run::command + ModifiedVerlet::setup/run (src/run.cpp:170-178, mvv_meso.cu:203-572) */
int mdpd_run(mdpd_t *h, int64_t nsteps);
/* ModifiedVerlet::setup only: rebuild, density pass, force pass (mvv_meso.cu:203-283) */
int mdpd_setup(mdpd_t *h);
/* steps without setup, thermo or output (the inner loop of ModifiedVerlet::run) */
int mdpd_step(mdpd_t *h, int64_t nsteps);
int mdpd_natoms(mdpd_t *h, int64_t *n);
/* state in tag order (row t-1 holds tag t): x,v 3*n doubles, tag/type n ints; NULL skips */
int mdpd_get_state(mdpd_t *h, double *x, double *v, int32_t *tag, int32_t *type, int64_t n);
/* replace positions/velocities (tag order); the next run/setup rebuilds */
int mdpd_set_state(mdpd_t *h, const double *x, const double *v, int64_t n);
/* compute temp/meso, pressure/meso, pe/meso (compute_temp_meso.cu:58-101,
 * compute_pressure_meso.cu:98-150, compute_pe_meso.cu:66) */
int mdpd_thermo(mdpd_t *h, mdpd_thermo_t *out);
/* thermo log accumulated so far (LAMMPS thermo lines) */
const char *mdpd_log(mdpd_t *h);
const char *mdpd_last_error(mdpd_t *h);
void mdpd_destroy(mdpd_t *h);

/* --- internal arrays for parity checks (internal particle order) ------------------------
 * name: "pos4" (float4, locals+ghosts), "vel4" (float4, locals+ghosts), "rho" (float,
 * locals+ghosts), "force" (float4, locals), "count" (int, locals), "tag" (int, locals),
 * "ghost_src" (int), "ghost_img" (int), "x" (double 3*n, locals, internal order),
 * "phi" (float, locals: wall volume fraction of fix aboundary/rho/meso),
 * "list" (int, n_col*ceil32(n): the transposed table, entry k of particle i at
 *   (i & ~31) * n_col + 32 k + (i & 31), like neigh_list_meso.cu:143-147 coalesced per warp; on an
 *   mDPD box without wall coupling or fix aboundary/meso its rows hold the owned pairs and those
 *   within r_d + skin + 1e-3, the rest of the reference's full list being unused there; the
 *   entries are particle indices: the device table's ownership flag in bit 31 is cleared).
 * sizes: returns the element count of a field in *count.                                 */
int mdpd_field_size(mdpd_t *h, const char *name, int64_t *count);
int mdpd_get_field(mdpd_t *h, const char *name, void *out, int64_t nbytes);
/* box geometry: lo[3], hi[3], cen[3], mbin[3] as doubles, cutneighmax, n_col, nghost,
 * n_bulk, nbuild (15 doubles) */
int mdpd_geometry(mdpd_t *h, double *out15);
/* neighbour pairs of the last build as (tag_i, tag_j), i local; *npairs on return */
int mdpd_get_pairs(mdpd_t *h, int32_t *tag_i, int32_t *tag_j, int64_t cap, int64_t *npairs);

/* --- pairwise RNG on explicit signature pairs (math_meso.h:465-473) --------------------- */
int mdpd_gaussian(const uint32_t *si, const uint32_t *sj, double *exact, float *fast, int64_t n);

/* --- build variant ------------------------------------------------------------------------ */
/* 1 when this library is the index-check build (libmdpd_check.so: `build.py --check`, compiled
 * with -DMDPD_CHECK), 0 for libmdpd.so.  The check build bounds-checks every neighbour, bin,
 * bucket and permutation index its kernels use; an index outside its array sets bit 64 of the
 * box's status word (mdpd_thermo_t.status), the access is skipped, and the run returns
 * MDPD_ERR_OVERFLOW naming the bit.  No reference counterpart: the reference only syncs and
 * gathers CUDA errors in its debug build (mvv_meso.cu:41-73). */
int mdpd_index_checks(void);

/* --- batched boxes: many independent boxes stepped by one graph per step ---------------- */
typedef struct mdpd_batch_s mdpd_batch_t;

typedef struct mdpd_box_spec {
    int32_t style;        /* 0 mdpd/meso, 1 dpd/meso */
    int32_t n;            /* particles */
    double lo[3], hi[3];
    double A, B, gamma, kT, cut, cut_r, cut_rho;  /* mdpd; dpd uses A (a0), gamma, cut, sigma */
    double sigma;         /* dpd only */
    double dt, skin, rho_est, mass;
    uint32_t seed;        /* pair RNG seed */
    int32_t every, delay, check;
    int32_t exact_rng;
    /* initial state (tag order, tags 1..n); when x is NULL the box is filled uniformly
     * at random from init_seed and v drawn from a Maxwell distribution at kT with zero
     * net momentum */
    const double *x, *v;
    uint64_t init_seed;
    double fill_lo[3], fill_hi[3];  /* random fill region (fill_hi <= fill_lo: whole box) */
    /* timestep the box starts at: 0 for a new run; a restart passes the step its state was
     * checkpointed at, so the pair RNG's step count (seed_now, pair_mdpd_meso.cu:295-297)
     * continues as after a LAMMPS restart file (atom_vec_mdpd_atomic_meso.cu:530-607) */
    int64_t start_step;
} mdpd_box_spec;

int mdpd_batch_create(mdpd_batch_t **b, const mdpd_box_spec *specs, int32_t nbox, const mdpd_opts *opts);
int mdpd_batch_setup(mdpd_batch_t *b);
/* nsteps steps of every box; the last one also computes pair energy and virial, so the thermo
 * read after the call (pressure, energy, virial, surface tension) is that step's, as the thermo
 * line at the end of a LAMMPS run (Run::command, run.cpp:170-178) */
int mdpd_batch_step(mdpd_batch_t *b, int64_t nsteps);
int mdpd_batch_thermo(mdpd_batch_t *b, int32_t box, mdpd_thermo_t *out);
/* every box's thermo in one pass (out[nbox], batch order; nbox must equal the batch's): the
 * per-box compute temp/pressure/pe/meso results (compute_temp_meso.cu:58-101,
 * compute_pressure_meso.cu:98-150) that mdpd_batch_thermo returns one at a time */
int mdpd_batch_thermo_all(mdpd_batch_t *b, mdpd_thermo_t *out, int32_t nbox);
int mdpd_batch_get_state(mdpd_batch_t *b, int32_t box, double *x, double *v, int64_t n);
/* every box's x and v at once (x[k], v[k]: 3 n_k doubles each in tag order, as mdpd_batch_get_state
 * writes them; a null x[k] or v[k] skips that array; nbox must equal the batch's): all boxes'
 * gathers and copies queued on the batch's stream with one wait at the end, instead of one host
 * round trip per box.  Pinned host arrays make each copy a direct DMA.  Device scratch of 6 n_max
 * doubles (the largest box) for the call, from the box pool. */
int mdpd_batch_get_states(mdpd_batch_t *b, double *const *x, double *const *v, int32_t nbox);
/* nsteps steps of every box, each step's thermo (every box, with that step's energy and virial:
 * a LAMMPS thermo line at every step, Run::command with thermo 1) written to
 * out[k * nbox + box], k = 0 .. nsteps-1.  Step k's thermo comes back to the host while step k+1
 * runs, through pinned staging the batch keeps, so the readback costs no device idle time.
 * *d2h_bytes_per_step (optional): device-to-host bytes copied per step.  A box's device error
 * bits seen in any step's thermo make the call return MDPD_ERR_NAN / MDPD_ERR_OVERFLOW after all
 * nsteps (the records still hold every step). */
int mdpd_batch_run_thermo(mdpd_batch_t *b, int64_t nsteps, mdpd_thermo_t *out, int64_t *d2h_bytes_per_step);
/* project autotuner: times the candidate shapes of the pair passes on this batch's current state
 * (each candidate's density and force passes evaluated once untimed and five times timed; they
 * recompute the same forces, so the boxes do not advance) and keeps the fastest. Pair-once mDPD
 * batches: *shape_density =
 * neighbour gathers in flight per lane in the density pass (4, 6 or 8); *shape_force = 32 (a
 * warp shares its 32 particles' pairs out to its 32 lanes, its compact rows staged in shared
 * memory first) or 0 (the same shares, each entry read from the table in the pair loop).
 * Full-list batches (classic DPD, wall-coupled mDPD): threads per particle of the density and
 * force passes (1, 2 or 4 each). */
int mdpd_batch_tune(mdpd_batch_t *b, int32_t *shape_density, int32_t *shape_force);
/* mdpd_batch_tune with its picks persisted in a JSON file (path; created when absent):
 * {"version": 1, "entries": {"<key>": {"density": D, "force": F, "ms_per_step": T}}} (T: the pick's pair
 * passes, ms per evaluation).  The key
 * names the workload class the pick applies to: GPU model and SM count, pass family and options,
 * mean density (0.25 steps), neighbour cutoff (0.05 steps), total particles and box count (powers
 * of two).  A stored key is applied without timing (*cached = 1); otherwise the batch is timed
 * as by mdpd_batch_tune and its pick added to the file (*cached = 0), which is rewritten
 * whole through a temporary and a rename, keeping the other members.  A malformed file or entry
 * returns MDPD_ERR_PARSE and is left untouched.  The reference's ThreadTuner learns online and
 * keeps nothing across runs (autotuner_meso.h:11-96). */
int mdpd_batch_tune_cached(mdpd_batch_t *b, const char *path, int32_t *shape_density, int32_t *shape_force,
                           int32_t *cached);
/* pin the pair-pass shapes (as mdpd_batch_tune reports them) without timing: one of the shapes
 * the batch's pass family offers, else MDPD_ERR_ARG.  No reference counterpart: the reference's
 * launch shapes come from its occupancy table (occupancy_meso.cu:8-50). */
int mdpd_batch_set_shapes(mdpd_batch_t *b, int32_t shape_density, int32_t shape_force);
/* last per-step device time in milliseconds measured with CUDA events over nsteps */
int mdpd_batch_time(mdpd_batch_t *b, int64_t nsteps, double *ms_per_step);
/* nsteps un-captured steps with CUDA events around each kernel group (same kernels as the
 * graph): per-step ms of [integrate, rebuild, density, force] and the number of steps whose
 * rebuild ran (5 doubles) */
int mdpd_batch_profile(mdpd_batch_t *b, int64_t nsteps, double *out5);
/* steps whose rebuild body ran since creation (device counter) */
int mdpd_batch_rebuild_steps(mdpd_batch_t *b, int64_t *n);
const char *mdpd_batch_last_error(mdpd_batch_t *b);
void mdpd_batch_destroy(mdpd_batch_t *b);

/* --- serving: admission by HBM budget, resident state, continuous batching -------------- */
typedef struct mdpd_server_s mdpd_server_t;

typedef struct mdpd_job_spec {
    mdpd_box_spec box;
    int64_t nsteps;
    int32_t keep_state;   /* keep the final x, v on the host for mdpd_server_get_state */
    int32_t pad;
} mdpd_job_spec;

typedef struct mdpd_job_result {
    int32_t state;        /* 0 queued, 1 running, 2 done, 3 failed, 4 cancelled, 5 preempted */
    int32_t error;        /* MDPD_* code when failed */
    int64_t steps_done;
    double submit_s, start_s, end_s;   /* host clock, seconds since server start */
    double step_ms_p50, step_ms_p99;   /* per-step latency of this job while resident */
    mdpd_thermo_t thermo;              /* at completion */
} mdpd_job_result;

/* device bytes a box of this spec holds while resident (the admission footprint) */
int mdpd_box_bytes(const mdpd_box_spec *spec, uint64_t *bytes);
/* starts the serving loop on opts->device. Before it returns, up to budget_bytes of device
 * memory (no more than is free, less 2 GiB) is mapped into the library's box pool, which keeps
 * it for the life of the process: admissions then take boxes without mapping fresh pages. */
int mdpd_server_start(mdpd_server_t **s, uint64_t budget_bytes, const mdpd_opts *opts);
int mdpd_server_submit(mdpd_server_t *s, const mdpd_job_spec *job, int64_t *job_id);
int mdpd_server_poll(mdpd_server_t *s, int64_t job_id, mdpd_job_result *out);
/* x, v (tag order, 3n each) of a done job kept with keep_state, or the checkpoint of a
 * preempted one; MDPD_ERR_STATE when there is none */
int mdpd_server_get_state(mdpd_server_t *s, int64_t job_id, double *x, double *v, int64_t n);
int mdpd_server_cancel(mdpd_server_t *s, int64_t job_id);
/* checkpoint and release a job (preemption, migration to another server or GPU): a running
 * job stops at the end of its current chunk of steps, its x, v are kept on the host and it
 * ends in state 5 with steps_done and thermo.step set; a queued one ends in state 5 at once,
 * its checkpoint the x, v it was submitted with (if any). Resubmitting the box with those
 * x, v, start_step = thermo.step and the remaining steps resumes it, as a run continued from
 * a LAMMPS restart file would (pack/unpack_restart, atom_vec_mdpd_atomic_meso.cu:530-607):
 * the same random-number steps, forces recomputed at setup from x and v (the integrator's
 * dissipative force then sees v at the full step once, where the running job had the half
 * step, so the continuation is statistically, not bitwise, the uninterrupted run) */
int mdpd_server_preempt(mdpd_server_t *s, int64_t job_id);
/* --- placement on the GPUs of a node ---------------------------------------------------------
 * Assigns independent boxes (a batch spread over devices) or jobs (servers on several devices)
 * to ndev devices: device_of[i] in [0, ndev), or -1 for an item that fits no device's
 * budget_bytes[d] (MDPD_ERR_BUDGET is then returned; the others are still placed).  Work is
 * specs[i].n * steps[i] (steps NULL: the particles, for boxes stepped together); items go in
 * decreasing work to the device with the least work so far among those with room (longest
 * processing time first; ties by index and by lower device), so every rank computes the same
 * placement from the same list and no data crosses devices.  work_per_device (optional, ndev):
 * the work placed on each.  Replaces the reference's static split of an ensemble into groups of
 * case_size ranks per case (main_ensemble, src/main.cpp:49-117). */
int mdpd_place(const mdpd_box_spec *specs, const int64_t *steps, int32_t nitem, int32_t ndev,
               const uint64_t *budget_bytes, int32_t *device_of, double *work_per_device);

/* JSON job specs: a file of boxes for one server,
 *   {"budget_gb": G, "timeout_s": T, "defaults": {<key>: value, ...},
 *    "jobs": [{"name": "a", "n": N, "box": L or [Lx, Ly, Lz], "steps": S, <key>: value, ...}]}
 * with a key per mdpd_box_spec field (style "mdpd"|"dpd", lo, A, B, gamma, kT, cut, cut_r,
 * cut_rho, sigma, dt, skin, rho_est, mass, seed, every, delay, check, exact_rng, init_seed,
 * fill_lo, fill_hi, start_step; unset ones take the mdpd/meso deck defaults).  An unknown key, a
 * value of the wrong kind, a missing n/box/steps or a box above the budget is MDPD_ERR_PARSE
 * naming the job and key, reported before any device work.
 * mdpd_jobs_validate: checks the file; the job count and the summed device footprint.
 * mdpd_run_jobs: submits every job to one server and waits for them (timeout_s, 0: no limit),
 * then writes to out_path (NULL: stdout) one JSON line per job in file order (state, steps,
 * queue and run seconds, particle-steps/s, p50/p99 step ms, builds, final temp/pe/press, status)
 * and a {"summary": ...} line with the server counters; returns the MDPD_* code of the first
 * job that did not finish, or MDPD_OK. */
int mdpd_jobs_validate(const char *spec_path, int32_t *njobs, uint64_t *bytes);
int mdpd_run_jobs(const char *spec_path, const char *out_path, const mdpd_opts *opts);
/* wait until every submitted job is done, failed or cancelled (timeout_s <= 0: no limit) */
int mdpd_server_drain(mdpd_server_t *s, double timeout_s);
/* the stepping set: between chunks the server steps, of its resident jobs, those with the least
 * remaining work (particles x steps left) up to n particles together (always at least one job);
 * the others wait on the device.  The set is picked again when a job of it ends, when a waiting
 * job fits beside it, or when a waiting job has less than half the remaining work of its longest
 * job.  n = 0 steps every resident job.  Default 8,388,608: a step over that many particles runs
 * near full throughput on a B200, and a short job that arrives behind long ones is done in its own
 * time.  No counterpart in the reference (one LAMMPS run per rank group, src/main.cpp:49-117). */
int mdpd_server_set_step_particles(mdpd_server_t *s, int64_t n);
/* where the serving loop's time went (8 doubles): host seconds creating boxes, forming batches
 * (work units and captured step graphs), setting up new boxes, running chunks; device seconds of
 * the chunks; number of batches formed; host seconds waiting with no job resident, and reading
 * states and retiring jobs after chunks */
int mdpd_server_timing(mdpd_server_t *s, double *out8);
/* throughput/latency summary: particle-steps/s, step p50/p99 ms, job p50/p99 s,
 * jobs done, peak resident bytes (7 doubles) */
int mdpd_server_stats(mdpd_server_t *s, double *out7);
void mdpd_server_stop(mdpd_server_t *s);

/* --- kinetic sums over caller-owned device arrays, allocating nothing -------------------
 * No counterpart in the reference. For callers that own all the device memory they want used
 * and call in from inside their own timestep (a LAMMPS fix/compute on its USER-MESO device
 * arrays, an application whose caching allocator or fixed arena holds the GPU): they cannot
 * let the library allocate, because cudaMalloc/cudaFree synchronise the whole device and fail
 * when the caller's pool holds the memory. This call uses no cudaMalloc, cudaFree or other
 * allocating routine; its scratch is a fixed 1.44 MB device array that every GPU loading the
 * library holds until the process exits.
 *   vx, vy, vz, mass: n doubles each, device memory of the current device (per-particle
 *   velocity components and mass, the layout of MesoAtomVec's dev_veloc(0..2) and dev_mass);
 *   mask: n ints on the device, or NULL to count every particle; a particle is counted when
 *   mask[i] & groupbit. stream: a cudaStream_t (NULL = the legacy default stream); the call
 *   returns after that stream has finished its work.
 *   sums (host, 11 doubles): sum m v^2, sum m v (x, y, z), sum m v_a v_b (xx yy zz xy xz yz),
 *   number of particles counted. Temperature in lj units is sums[0] / (3 sums[10] - 3).
 *   err (optional, err_len bytes): the reason for a non-zero return.
 * Limit: n <= 16,777,216 (2^24) per call; larger n returns MDPD_ERR_ARG without launching.
 * The first call on each device looks up the scratch array's device address with that device
 * current and keeps it for the life of the process; after a cudaDeviceReset of that device the
 * kept address is stale, so a host that resets a device must not call this again in the same
 * process. Every call copies the sums to pageable host memory and synchronises its stream: no
 * call may be made while its stream (or, in global capture mode, any stream) is being captured,
 * and one made on a capturing stream returns MDPD_ERR_ARG without launching. Every call on a
 * device shares the one scratch array: calls whose work overlaps on the GPU (two host threads on two
 * streams, say) race and can return wrong sums, so run them one after another. Nothing needs
 * clearing between calls: each call writes every scratch entry it reads. */
int mdpd_kinetic_sums_noalloc(const double *vx, const double *vy, const double *vz,
                              const double *mass, const int32_t *mask, int32_t groupbit,
                              int64_t n, void *stream, double *sums, char *err, int64_t err_len);

#ifdef __cplusplus
}
#endif
#endif
