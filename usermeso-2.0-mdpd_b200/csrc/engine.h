// Host runtime of the B200 DPD/mDPD timestep path: device-resident boxes, batches of
// boxes stepped by one captured CUDA graph per step, thermo reductions.
#pragma once

#include <functional>

#include <nvtx3/nvToolsExt.h>
#include <cstdint>
#include <string>
#include <vector>

#include "kernels.h"

namespace mdpd {

// physics + geometry of one box, in reference units (LAMMPS lj)
struct PairParam {
    int set = 0;
    double cut = 0, cut_r = 0, A = 0, B = 0, gamma = 0, sigma = 0, expw = 1;
};

struct Spec {
    int style = 0;  // 0 mdpd/meso, 1 dpd/meso
    int ntype = 1;
    double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    double skin = 0.3;
    int every = 1, delay = 0, check = 1;
    double dt = 0.01;
    double kT = 1.0;       // mdpd: sigma = sqrt(2 kT gamma)
    uint32_t seed = 1;
    double rho_est = 0;    // atom_style mdpd/atomic/meso density estimate (0: nlocal/volume)
    PairParam pair[kMaxTypes][kMaxTypes];
    double mass[kMaxTypes] = {1, 1, 1, 1, 1, 1, 1, 1};
    int nve_bit = 1;       // group bitmask of fix nve/meso
    int rho_bit = 1;       // group bitmask of fix aboundary/rho/meso
    double cut_rho = 0.75;
    int body_bit = 0;
    double body[3] = {0, 0, 0};
    int arb_bc = 0, mobile_bit = 0, wall_bit = 0;  // pair_style ... fluid_group wall_group
    int wall_fix = 0;                              // aboundary wall/mobile given
    double cut_phi = 0, rho_wall = 0, phi_c = 0;
    // fix aboundary/meso (fix_aboundary_meso.cu:31-82): group, wall group, rho, sigma
    int ab_mobile_bit = 0, ab_wall_bit = 0;
    double ab_rho0 = 0, ab_sigma = 0;
    int exact_rng = 0;
    double ghost_factor = 1.0;   // ghost capacity multiplier
    long long step0 = 0;         // timestep the box starts at (a restart continues the RNG's steps)
};

struct Particles {
    std::vector<double> x, v;        // 3 per particle
    std::vector<int32_t> tag, type, mask;
    size_t size() const { return tag.size(); }
};

struct Thermo {
    long long step = 0, nbuild = 0;
    double ke_all = 0, ke_group = 0, pe = 0, virial[6] = {0, 0, 0, 0, 0, 0}, mom[3] = {0, 0, 0};
    double ke_tensor[6] = {0, 0, 0, 0, 0, 0};
    double temp = 0, press = 0;
    double ptensor[6] = {0, 0, 0, 0, 0, 0};  // (kinetic + virial) / V, xx yy zz xy xz yz
    double surface_tension = 0;              // (Lx/2)(Pxx - (Pyy+Pzz)/2), slab normal to x
    int n = 0, n_group = 0;
    int status = 0;
};

// a box filled on the device: positions uniform in [lo, hi) (a position that reaches the box's
// hi folds to its lo), velocities Maxwell with standard deviation vscale per component and zero
// net momentum, both from a counter-based hash of (seed, particle, component)
struct Fill {
    double lo[3], hi[3];
    uint64_t seed;
    double vscale;
};

class Box {
public:
    Box(const Spec &spec, const Particles &p, int sms);
    Box(const Spec &spec, int n, const Fill &fill, int sms, bool wait = true);
    // from caller arrays (AoS x[3n], v[3n]; v null: at rest; tag/type/mask null: tags 1..n,
    // type 1, mask 1), copied straight to the device without host staging. wait = false leaves
    // the copies queued on the legacy default stream: the caller synchronises it before it
    // lets go of the arrays (a batch of boxes waits once, not once per box)
    Box(const Spec &spec, int n, const double *x, const double *v, const int32_t *tag, const int32_t *type,
        const int32_t *mask, int sms, bool wait = true);
    ~Box();
    Box(const Box &) = delete;
    Box &operator=(const Box &) = delete;

    BoxDesc desc;       // host copy of the device descriptor (pointers + parameters)
    BoxState *d_state;  // device scalars
    Spec spec;
    int n = 0;
    int nbin = 0;
    size_t bytes = 0;   // device memory held
    int n_group = 0;

    static size_t estimate_bytes(const Spec &spec, int n);

    // host views (synchronous)
    BoxState state() const;
    void download_state(double *x, double *v, double *f, int32_t *tag, int32_t *type,
                        int32_t *mask) const;           // current internal order
    void upload_xv(const double *x, const double *v);  // by tag, host order of tags 1..n
    // positions and velocities in tag order (tags 1..n), gathered on the device and copied
    // straight into x[3n] and v[3n] (either may be null)
    // scratch: device memory of at least 48 n bytes (null: allocated and freed by the call)
    void download_by_tag(double *x, double *v, double *scratch = nullptr) const;

private:
    // every device array of the box lives in one allocation: layout() runs twice, first to
    // size the arena (alloc returns null), then to hand out 256-byte aligned pieces of it
    char *arena_ = nullptr;
    size_t arena_need_ = 0, arena_off_ = 0;
    void layout(const Spec &s, int na);
    void release() noexcept;  // returns the arena to the pool
    void init(const Spec &s, const double *x, const double *v, const int32_t *tag, const int32_t *type,
              const int32_t *mask, bool wait = true, const Fill *fill = nullptr);
    template <class T> T *alloc(size_t count);
};

// A set of boxes stepped together; one box is the plain single-box path.
class Batch {
public:
    Batch(std::vector<Box *> boxes, const StepConfig &cfg);
    ~Batch();
    Batch(const Batch &) = delete;
    Batch &operator=(const Batch &) = delete;

    void setup();                          // forced rebuild, density, force (no kick), thermo partials
    // setup of the listed boxes only: rebuild, density and force passes over their units (the
    // other boxes keep their state and forces)
    void setup_boxes(const std::vector<int> &which);
    void reconfigure(const StepConfig &c);  // new pair-pass shapes: recapture the step graphs
    // nsteps graph replays; with ev_last the last one also computes energy and virial (the
    // step a thermo line reports, as at the end of a LAMMPS run)
    void run(long long nsteps, bool sync = true, bool ev_last = false);
    void step_ev();                        // one step with energy/virial (thermo step)
    // nsteps un-captured steps with CUDA events around each kernel group; per-step averages
    // in ms: [integrate, rebuild (all steps), density, force], plus steps that rebuilt
    void profile(long long nsteps, double out[5]);
    // device ms of one evaluation of the pair passes (density, force without a kick) on the
    // current state, averaged over reps after one untimed: the passes recompute the same forces,
    // so the boxes do not advance (the autotuner's timing)
    double time_pair_passes(int reps);
    long long rebuild_steps();             // steps whose rebuild body ran (device counter)
    void thermo(std::vector<Thermo> &out); // reduce + download (synchronous)
    // nsteps steps, each with energy and virial and followed by its thermo; sink(k, thermo) gets
    // step k's every-box thermo while step k + 1 runs (pinned double-buffered staging)
    void run_thermo(long long nsteps, const std::function<void(long long, const std::vector<Thermo> &)> &sink);
    size_t thermo_bytes_per_step() const;  // device-to-host bytes run_thermo copies per step
    int status(std::string &msg);          // OR of box status words
    void read_states(std::vector<BoxState> &out);  // every box's device scalars, one copy
    // every box's x, v in tag order into x[k], v[k] (null: skipped): each box's gather and
    // copies queued on the batch's stream through one scratch of the largest box, one wait
    void download_all(double *const *x, double *const *v);
    cudaStream_t stream() const { return stream_; }
    const std::vector<Box *> &boxes() const { return boxes_; }
    StepConfig cfg;
    BatchUnits units;
    BoxDesc *d_boxes = nullptr;

private:
    std::vector<Box *> boxes_;
    cudaStream_t stream_ = nullptr;
    int *d_done = nullptr;
    double *d_thermo = nullptr;
    BoxState *d_states = nullptr;  // gathered copies of the boxes' scalars
    std::vector<Unit *> unit_allocs_;
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};  // [ev]
    cudaGraph_t graph_src_[2] = {nullptr, nullptr};
    char *h_stage_ = nullptr;                    // run_thermo's pinned staging, two slots
    cudaEvent_t ev_stage_[2] = {nullptr, nullptr};
    void to_thermo(const double *partials, const BoxState *states, std::vector<Thermo> &out) const;
    void build_units();
    void capture(int ev);
};

// an NVTX range over a host scope: the phases of setup, stepping, rebuild and I/O show by name on
// an Nsight timeline, and `ncu --nvtx --nvtx-include "<name>/"` selects the kernels launched in
// one (a push and a pop, nanoseconds, when no tool is attached)
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

std::string status_text(int bits);  // names of the set bits of a box status word
std::string cuda_err(cudaError_t e);
void check_cuda(cudaError_t e, const char *what);
// AoS x[3n], v[3n] of a Fill on the device (stream s); mom: 3 zeroed words of device scratch
void launch_fill(cudaStream_t s, const Fill &f, const double box_lo[3], const double box_hi[3], int n, double *xa,
                 double *va, unsigned long long *mom);
int sm_count();
// maps up to `bytes` of device memory into the current device's box pool ahead of use (halving
// the request until it fits, down to 1 GiB); returns the bytes reserved (0: none)
size_t reserve_box_pool(size_t bytes);

}  // namespace mdpd
