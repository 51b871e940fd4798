// Host runtime: device allocation of boxes, the per-step CUDA graph (integrate ->
// IF(rebuild){...} -> density -> force), setup and thermo.
#include "engine.h"

#include <functional>

#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>

namespace mdpd {

std::string cuda_err(cudaError_t e) { return std::string(cudaGetErrorName(e)) + ": " + cudaGetErrorString(e); }

void check_cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA ") + what + ": " + cuda_err(e));
}

int sm_count()
{
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n;
}

static int ceil_to(int x, int inc) { return ((x + inc - 1) / inc) * inc; }

struct Geometry {
    double prd[3], cen[3], cutneighmax, cutghost, binsize[3], bininv[3];
    int mbin[3], n_col, n_col2;
    float rc2_tail, rc2_force;
};

static Geometry geometry(const Spec &s, int n)
{
    // neighbor.cpp:258-268, neighbor_meso.cu:771-853, neigh_list_meso.cu:78-90
    Geometry g{};
    double cutforce = 0;
    for (int i = 0; i < s.ntype; ++i)
        for (int j = 0; j < s.ntype; ++j) cutforce = std::max(cutforce, s.pair[i][j].cut);
    g.cutneighmax = cutforce + s.skin;
    g.cutghost = g.cutneighmax;
    for (int d = 0; d < 3; ++d) {
        g.prd[d] = s.hi[d] - s.lo[d];
        g.cen[d] = 0.5 * (s.hi[d] + s.lo[d]);
    }
    const double vol = g.prd[0] * g.prd[1] * g.prd[2];
    const double dens = s.rho_est > 0 ? s.rho_est : n / vol;
    double e = dens * (4.0 / 3.0 * 3.142 * std::pow(g.cutneighmax, 3.0));
    e *= 4.0;
    e = std::max(e, 32.0);
    g.n_col = ceil_to((int)e, 32);
    const double inv_opt = 1.0 / g.cutneighmax;
    for (int d = 0; d < 3; ++d) {
        const int nb = std::max((int)(g.prd[d] * inv_opt), 1);
        g.mbin[d] = nb + 2;
        g.binsize[d] = g.prd[d] / nb;
        g.bininv[d] = 1.0 / g.binsize[d];
    }
    g.rc2_tail = (float)std::pow(g.cutneighmax, 2.0);
    double e2 = dens * (4.0 / 3.0 * 3.142 * std::pow(cutforce, 3.0)) * 4.0 * 0.5;  // half list
    e2 = std::max(e2, 32.0);
    g.n_col2 = ceil_to((int)e2, 32);
    g.rc2_force = (float)(cutforce * cutforce);
    return g;
}

static long long ghost_estimate(const Spec &s, const Geometry &g, int n)
{
    double f = 1.0;
    for (int d = 0; d < 3; ++d) f *= 1.0 + 2.0 * g.cutghost / g.prd[d];
    const double est = (f - 1.0) * n;
    return (long long)(est * 1.5 * s.ghost_factor) + 4096;
}

size_t Box::estimate_bytes(const Spec &spec, int n)
{
    const Geometry g = geometry(spec, n);
    const long long nbin = (long long)g.mbin[0] * g.mbin[1] * g.mbin[2];
    const long long gc = ghost_estimate(spec, g, n);
    const long long nrow = ceil_to(n, 32);
    size_t b = 0;
    b += (size_t)n * (2 * 6 * 8 + 3 * 8 + 2 * 16 + 6 * 4 + 2 * 4 + 3 * 4 + 4);  // x,v,xh,f,tag/type/mask,phi,cls,sub,perm,count
    b += (size_t)(n + gc) * (16 + 16 + 4 + 4 + 4 + 16 + 4);                      // pos, vel, rho, bin_of, bin_order, bpos, gfirst
    b += (size_t)gc * 8;
    b += (size_t)nrow * g.n_col * 4;
    if (spec.style == 0) b += (size_t)nrow * (g.n_col2 + 1) * 4 + (size_t)n * 24 + (size_t)(n + gc) * 16;
    b += (size_t)nbin * (4 + 3 * 4) * 3;
    b += (size_t)((n + kUnit - 1) / kUnit) * kPartialStride * 8;
    return b + (1u << 20);
}

// Box arenas come from one stream-ordered pool per device that keeps freed memory mapped, so
// boxes created after others were destroyed (a batch rebuilt by the server, a new batch after an
// old one) do not pay for mapping fresh pages again. The pool is created on first use with the
// device that is current.
static cudaMemPool_t box_pool()
{
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "device");
    if (dev < 0 || dev >= 64) throw std::runtime_error("CUDA device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        check_cuda(cudaMemPoolCreate(&pools[dev], &props), "memory pool");
        uint64_t keep = UINT64_MAX;
        check_cuda(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep), "memory pool");
    }
    return pools[dev];
}

// A box's arena is allocated, and the caller's x and v copied into it, on an upload stream of
// the device (one per device, kept for the process); the legacy stream, which zeroes the arena
// and runs the box's set-up kernels, waits for those copies. Boxes created one after another
// then keep the copy engine busy: one box's copies overlap the previous box's kernels.
static cudaStream_t upload_stream()
{
    static std::mutex mu;
    static cudaStream_t streams[64] = {};
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "device");
    if (dev < 0 || dev >= 64) throw std::runtime_error("CUDA device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!streams[dev]) check_cuda(cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking), "upload stream");
    return streams[dev];
}

size_t reserve_box_pool(size_t bytes)
{
    // one allocation of the whole size, freed back at once: the pool keeps the memory mapped
    // (release threshold: never), so boxes created later take it without mapping new pages
    cudaMemPool_t pool = box_pool();
    cudaStream_t s;
    check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
    size_t got = 0;
    for (size_t want = bytes; want >= (size_t(1) << 30); want /= 2) {
        void *p = nullptr;
        if (cudaMallocFromPoolAsync(&p, want, pool, s) == cudaSuccess) {
            check_cuda(cudaFreeAsync(p, s), "pool reserve");
            got = want;
            break;
        }
        cudaGetLastError();  // an out-of-memory answer is not left for the next caller
    }
    check_cuda(cudaStreamSynchronize(s), "pool reserve");
    cudaStreamDestroy(s);
    return got;
}

// a batch's own small arrays (box table, work units, counters) come from the box pool on the
// batch's stream and go back to it stream-ordered: cudaMalloc/cudaFree here took up to ~1 s per
// batch on a device whose pool holds a large mapped budget, which a server forming a batch for
// each change of its stepping set paid every time
template <class T> static T *batch_alloc(size_t count, cudaStream_t s)
{
    void *p = nullptr;
    check_cuda(cudaMallocFromPoolAsync(&p, sizeof(T) * std::max<size_t>(count, 1), box_pool(), s), "batch arrays");
    return static_cast<T *>(p);
}

template <class T> T *Box::alloc(size_t count)
{
    const size_t bytes_ = (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~size_t(255);
    if (!arena_) {
        arena_need_ += bytes_;
        return nullptr;
    }
    T *p = reinterpret_cast<T *>(arena_ + arena_off_);
    arena_off_ += bytes_;
    return p;
}

void Box::layout(const Spec &s, int na)
{
    BoxDesc &B = desc;
    // the host-initialised arrays first, contiguous, so one copy uploads them all
    for (int d = 0; d < 3; ++d) B.x[0][d] = alloc<double>(n);
    for (int d = 0; d < 3; ++d) B.v[0][d] = alloc<double>(n);
    for (int d = 0; d < 3; ++d) B.xh[d] = alloc<double>(n);
    B.tag[0] = alloc<int>(n);
    B.type[0] = alloc<int>(n);
    B.mask[0] = alloc<int>(n);
    for (int d = 0; d < 3; ++d) {
        B.x[1][d] = alloc<double>(n);
        B.v[1][d] = alloc<double>(n);
    }
    B.tag[1] = alloc<int>(n);
    B.type[1] = alloc<int>(n);
    B.mask[1] = alloc<int>(n);
    for (int c = 0; c < 2; ++c) {
        B.f[c] = alloc<float4>(n);
        B.phi[c] = alloc<float>(n);
    }
    B.pos = alloc<float4>(na);
    B.vel = alloc<float4>(na);
    B.rho = alloc<float>(na);
    B.gsrc = alloc<int>(B.ghost_cap);
    B.gimg = alloc<int>(B.ghost_cap);
    B.gfirst = alloc<int>(n + 1);
    B.count = alloc<int>(B.nrow);
    B.table = alloc<int>((size_t)B.nrow * B.n_col);
    if (s.style == 0) {
        B.count2 = alloc<int>(B.nrow);
        B.table2 = alloc<int>((size_t)B.nrow * B.n_col2);
        B.facc = alloc<unsigned long long>(3 * (size_t)n);
        B.posrho = alloc<float4>(na);
    }
    B.bin_rank = alloc<int>(nbin);
    B.cls_count = alloc<int>(2 * (size_t)nbin + 1);
    B.cls_start = alloc<int>(2 * (size_t)nbin + 1);
    B.cls_cursor = alloc<int>(2 * (size_t)nbin + 1);
    B.cls_of = alloc<int>(n);
    B.sub_of = alloc<int>(n);
    B.perm = alloc<int>(n);
    B.bin_of = alloc<int>(na);
    B.bin_count = alloc<int>(nbin + 1);
    B.bin_start = alloc<int>(nbin + 1);
    B.bin_cursor = alloc<int>(nbin + 1);
    B.bin_order = alloc<int>(na);
    B.bpos = alloc<float4>(na);
    const int nchunk = std::max({2 * nbin, n + 1, nbin}) / kScanChunk + 2;
    B.scan_part = alloc<int>(nchunk);
    B.partial = alloc<double>((size_t)((n + kUnit - 1) / kUnit) * kPartialStride);
    d_state = alloc<BoxState>(1);
    B.st = d_state;
}

Box::Box(const Spec &s, const Particles &p, int sms) : spec(s)
{
    Range r("mdpd::box_create");
    (void)sms;
    n = (int)p.size();
    try {
        init(s, p.x.data(), p.v.data(), p.tag.data(), p.type.data(), p.mask.data());
    } catch (...) {
        release();  // a constructor that throws runs no destructor
        throw;
    }
}

Box::Box(const Spec &s, int n_, const double *x, const double *v, const int32_t *tag, const int32_t *type,
         const int32_t *mask, int sms, bool wait)
    : spec(s)
{
    Range r("mdpd::box_create");
    (void)sms;
    n = n_;
    try {
        init(s, x, v, tag, type, mask, wait);
    } catch (...) {
        release();
        throw;
    }
}

Box::Box(const Spec &s, int n_, const Fill &fill, int sms, bool wait) : spec(s)
{
    Range r("mdpd::box_create");
    (void)sms;
    n = n_;
    try {
        init(s, nullptr, nullptr, nullptr, nullptr, nullptr, wait, &fill);
    } catch (...) {
        release();
        throw;
    }
}

void Box::init(const Spec &s, const double *x, const double *v, const int32_t *tag, const int32_t *type,
               const int32_t *mask, bool wait, const Fill *fill)
{
    if (n <= 0) throw std::runtime_error("ARG: box has no particles");
    if (s.ntype < 1 || s.ntype > kMaxTypes) throw std::runtime_error("ARG: 1..8 atom types supported");
    for (int a = 0; a < s.ntype; ++a)
        for (int b = 0; b < s.ntype; ++b)
            if (!s.pair[a][b].set) throw std::runtime_error("PARSE: All pair coeffs are not set");
    const Geometry g = geometry(s, n);
    for (int d = 0; d < 3; ++d)
        if (g.mbin[d] - 2 < 3)
            throw std::runtime_error("ARG: box edge shorter than 3 x (cutoff + skin) is not supported");
    std::memset(&desc, 0, sizeof(desc));
    BoxDesc &B = desc;
    for (int d = 0; d < 3; ++d) {
        B.lo[d] = s.lo[d];
        B.hi[d] = s.hi[d];
        B.prd[d] = g.prd[d];
        B.cen[d] = g.cen[d];
        B.binsize[d] = g.binsize[d];
        B.bininv[d] = g.bininv[d];
        B.coord_inv[d] = 16 * g.bininv[d];
        B.mbin[d] = g.mbin[d];
    }
    B.cutghost = g.cutghost;
    B.triggersq = 0.25 * s.skin * s.skin;
    B.rc2_tail = g.rc2_tail;
    B.rc2_force = g.rc2_force;
    {
        const double rn = s.cut_rho + s.skin + 1e-3;
        B.rn2_list = (float)(rn * rn);
        B.list_reduce = 0;
    }
    B.ab_mobile_bit = s.ab_mobile_bit;
    B.ab_wall_bit = s.ab_wall_bit;
    B.ab_rho0 = (float)s.ab_rho0;
    B.ab_sigma = (float)s.ab_sigma;
    // 1 / sqrt((2 pi)^3 sigma^3), the Gaussian's normalisation (fix_aboundary_meso.cu:275)
    B.ab_nfactor = s.ab_mobile_bit ? (float)(1.0 / std::sqrt(std::pow(2 * M_PI, 3.0) * std::pow(s.ab_sigma, 3.0))) : 0.f;
    B.n_col2 = g.n_col2;
    nbin = B.nbin = g.mbin[0] * g.mbin[1] * g.mbin[2];
    B.nlocal = n;
    B.nrow = ceil_to(n, 32);
    B.ghost_cap = (int)std::min<long long>(ghost_estimate(s, g, n), 8LL * n + 4096);
    B.n_col = g.n_col;
    B.fix_pair_max = (float)(2147483648.0 / (double)(g.n_col + 1));
    B.every = std::max(1, s.every);
    B.delay = s.delay;
    B.check = s.check;
    B.style = s.style;
    B.ntype = s.ntype;
    B.exact_rng = s.exact_rng;
    for (int a = 0; a < s.ntype; ++a)
        for (int b = 0; b < s.ntype; ++b) {
            const PairParam &q = s.pair[a][b];
            PairCoeff &c = B.coeff[a * s.ntype + b];
            c.cut = (float)q.cut;
            c.cutsq = (float)(q.cut * q.cut);
            c.inv_cut = (float)(1.0 / q.cut);
            c.cut_r = (float)q.cut_r;
            c.inv_cut_r = q.cut_r > 0 ? (float)(1.0 / q.cut_r) : 0.f;
            c.A = (float)q.A;
            c.B = (float)q.B;
            c.gamma = (float)q.gamma;
            // mdpd: sigma = sqrt(2 kB T gamma) (pair_mdpd_meso.cu:387); dpd: given
            c.sigma = (float)(s.style == 0 ? std::sqrt(2.0 * s.kT * q.gamma) : q.sigma);
            c.expw = (float)q.expw;
            c.e_cut = (float)(0.5 * q.A * q.cut);
            c.e_cut_r = (float)(0.5 * q.B * q.cut_r);
        }
    const double dtf = 0.5 * s.dt;  // ftm2v = 1 (units lj)
    for (int t = 0; t < kMaxTypes; ++t) {
        B.mass[t] = s.mass[t];
        B.dtfm[t] = dtf * rcp_newton(s.mass[t]);
    }
    B.dtv = s.dt;
    B.dtf = dtf;
    B.dt_inv_sqrt = (float)(1.0 / std::sqrt(s.dt));
    B.seed = s.seed;
    B.nve_bit = s.nve_bit;
    B.rho_bit = s.rho_bit;
    B.cut_rho = (float)s.cut_rho;
    B.rho_factor = 15.0 / (2.0 * M_PI * s.cut_rho * s.cut_rho * s.cut_rho * s.cut_rho * s.cut_rho);
    B.body_bit = s.body_bit;
    for (int d = 0; d < 3; ++d) B.body[d] = s.body[d];
    B.arb_bc = s.arb_bc;
    B.mobile_bit = s.mobile_bit;
    B.wall_bit = s.wall_bit;
    B.wall_fix = s.wall_fix;
    B.cut_phi = (float)s.cut_phi;
    if (s.wall_fix) {
        const double rc7 = std::pow(s.cut_phi, 7.0);
        B.phi_factor = (float)(105.0 / (16.0 * M_PI * s.rho_wall * rc7));
        B.dw_factor = (float)(-315.0 / (4.0 * M_PI * s.rho_wall * rc7));
        B.phi_c = (float)s.phi_c;
    }

    const int na = n + B.ghost_cap;
    // the pair-once compact table packs j (27 bits) and j's type (3 bits) into one word
    if (s.style == 0 && (long long)na >= (1LL << 27))
        throw std::runtime_error("ARG: box too large for one device box: " + std::to_string(na) +
                                 " particles and ghost images (limit 134217727)");
    // the list kernels address the table with unsigned 32-bit offsets
    if ((long long)B.nrow * B.n_col > 0xffffffffLL)
        throw std::runtime_error("ARG: box too large for one device box: " + std::to_string(n) + " particles need " +
                                 std::to_string((long long)B.nrow * B.n_col) +
                                 " neighbour-table entries (limit 4294967295); split it into boxes");
    layout(s, na);  // size the arena
    if (!x && !fill) throw std::runtime_error("ARG: no positions");
    const cudaStream_t up = upload_stream();
    {
        void *a = nullptr;
        const cudaError_t e = cudaMallocFromPoolAsync(&a, arena_need_, box_pool(), up);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("OOM: device allocation of " + std::to_string(arena_need_) + " bytes failed");
        }
        arena_ = static_cast<char *>(a);
    }
    layout(s, na);  // hand out the pieces
    // the caller's AoS x and v go to the list table's space (unused until the first build, which
    // writes every entry it later reads) on the upload stream; the legacy stream waits for them
    // before anything of its own touches the arena
    const size_t stage_need = 6 * sizeof(double) * (size_t)n;
    double *sx = reinterpret_cast<double *>(B.table), *sv = sx + 3 * (size_t)n;
    {
        if ((size_t)B.nrow * B.n_col * sizeof(int) < stage_need) {
            cudaFreeAsync(arena_, up);
            arena_ = nullptr;
            throw std::runtime_error("ARG: list table too small to stage");
        }
        if (!fill) {
            check_cuda(cudaMemcpyAsync(sx, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, up), "upload");
            if (v) check_cuda(cudaMemcpyAsync(sv, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, up), "upload");
        }
        cudaEvent_t ev;
        check_cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "upload event");
        check_cuda(cudaEventRecord(ev, up), "upload event");
        check_cuda(cudaStreamWaitEvent(0, ev, 0), "upload event");
        check_cuda(cudaEventDestroy(ev), "upload event");
    }
    {
        // zero everything but the neighbour tables (most of the arena): every build writes each
        // list entry it later reads, and each density pass each compact entry
        auto zero = [&](const void *from, const void *to) {
            const char *a = static_cast<const char *>(from), *b = static_cast<const char *>(to);
            if (b > a) check_cuda(cudaMemsetAsync(const_cast<char *>(a), 0, (size_t)(b - a), 0), "memset");
        };
        const char *end = arena_ + arena_need_;
        const char *t1 = reinterpret_cast<const char *>(desc.table), *t1e = t1 + sizeof(int) * (size_t)desc.nrow * desc.n_col;
        if (desc.table2) {
            const char *t2 = reinterpret_cast<const char *>(desc.table2);
            const char *t2e = t2 + sizeof(int) * (size_t)desc.nrow * desc.n_col2;
            zero(arena_, t1);
            zero(t1e, t2);
            zero(t2e, end);
        } else {
            zero(arena_, t1);
            zero(t1e, end);
        }
    }
    if (s.step0 != 0) {  // a restarted box: its step counter continues (after the memset, same stream)
        BoxState st{};
        st.step = s.step0;
        check_cuda(cudaMemcpy(d_state, &st, sizeof(st), cudaMemcpyHostToDevice), "state");
    }
    bytes = arena_need_;

    // Morton rank of every bin: reorder buckets are visited in Morton order of their bin
    launch_bin_ranks(0, g.mbin, B.bin_rank);
    // initial state into buffer 0: the staged x and v (or a device fill of them), split by a
    // kernel into x, xh and v components, which also fills tags/types/masks that were not given
    {
        if (fill) {
            // the thermo partials (zeroed with the arena, rewritten by every thermo pass) hold
            // the fill's momentum sum
            launch_fill(0, *fill, s.lo, s.hi, n, sx, sv, reinterpret_cast<unsigned long long *>(B.partial));
            v = sv;  // non-null: the split kernel takes the filled velocities
        }
        if (tag) check_cuda(cudaMemcpyAsync(B.tag[0], tag, sizeof(int) * n, cudaMemcpyHostToDevice, 0), "upload");
        if (type) check_cuda(cudaMemcpyAsync(B.type[0], type, sizeof(int) * n, cudaMemcpyHostToDevice, 0), "upload");
        if (mask) check_cuda(cudaMemcpyAsync(B.mask[0], mask, sizeof(int) * n, cudaMemcpyHostToDevice, 0), "upload");
        launch_load_state(0, sx, v ? sv : nullptr, n, B.x[0], B.xh, B.v[0], tag ? nullptr : B.tag[0],
                          type ? nullptr : B.type[0], mask ? nullptr : B.mask[0]);
        check_cuda(cudaGetLastError(), "upload");
        if (wait) check_cuda(cudaStreamSynchronize(0), "upload");
        if (mask) {
            for (int i = 0; i < n; ++i)
                if (mask[i] & s.nve_bit) ++n_group;
        } else {
            n_group = (1 & s.nve_bit) ? n : 0;
        }
    }
}

Box::~Box() { release(); }

void Box::release() noexcept
{
    if (!arena_) return;
    cudaDeviceSynchronize();  // no kernel of any stream may still use the arena
    cudaFreeAsync(arena_, 0);
    cudaStreamSynchronize(0);
    arena_ = nullptr;
}

// both buffers of a box's x, v and tags: the tag gather picks the live one on the device
static StateBuffers state_buffers(const BoxDesc &desc)
{
    StateBuffers sb;
    for (int c = 0; c < 2; ++c) {
        for (int k = 0; k < 3; ++k) sb.x[c][k] = desc.x[c][k], sb.v[c][k] = desc.v[c][k];
        sb.tag[c] = desc.tag[c];
    }
    return sb;
}

void Box::download_by_tag(double *x, double *v, double *scratch) const
{
    Range r("mdpd::download");
    double *d = scratch;
    if (!d) d = batch_alloc<double>(6 * (size_t)n, 0);  // the box pool, stream-ordered
    // the gather picks the live buffer on the device: one wait per call, at the end
    launch_gather_by_tag(0, state_buffers(desc), desc.st, n, d, d + 3 * (size_t)n);
    check_cuda(cudaGetLastError(), "download");
    if (x) check_cuda(cudaMemcpyAsync(x, d, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, 0), "download");
    if (v) check_cuda(cudaMemcpyAsync(v, d + 3 * (size_t)n, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, 0),
                      "download");
    check_cuda(cudaStreamSynchronize(0), "download");
    if (!scratch) cudaFreeAsync(d, 0);
}

BoxState Box::state() const
{
    BoxState st;
    check_cuda(cudaMemcpy(&st, d_state, sizeof(st), cudaMemcpyDeviceToHost), "download state");
    return st;
}

void Box::download_state(double *x, double *v, double *f, int32_t *tag, int32_t *type, int32_t *mask) const
{
    const BoxState st = state();
    const int c = st.cur;
    std::vector<double> col(n);
    for (int d = 0; d < 3; ++d) {
        if (x) {
            check_cuda(cudaMemcpy(col.data(), desc.x[c][d], sizeof(double) * n, cudaMemcpyDeviceToHost), "download");
            for (int i = 0; i < n; ++i) x[3 * i + d] = col[i];
        }
        if (v) {
            check_cuda(cudaMemcpy(col.data(), desc.v[c][d], sizeof(double) * n, cudaMemcpyDeviceToHost), "download");
            for (int i = 0; i < n; ++i) v[3 * i + d] = col[i];
        }
    }
    if (f) {
        std::vector<float4> ff(n);
        check_cuda(cudaMemcpy(ff.data(), desc.f[c], sizeof(float4) * n, cudaMemcpyDeviceToHost), "download");
        for (int i = 0; i < n; ++i) {
            f[3 * i] = ff[i].x;
            f[3 * i + 1] = ff[i].y;
            f[3 * i + 2] = ff[i].z;
        }
    }
    if (tag) check_cuda(cudaMemcpy(tag, desc.tag[c], sizeof(int) * n, cudaMemcpyDeviceToHost), "download");
    if (type) check_cuda(cudaMemcpy(type, desc.type[c], sizeof(int) * n, cudaMemcpyDeviceToHost), "download");
    if (mask) check_cuda(cudaMemcpy(mask, desc.mask[c], sizeof(int) * n, cudaMemcpyDeviceToHost), "download");
}

void Box::upload_xv(const double *x, const double *v)
{
    // x, v given in tag order (tag t at row t-1); scattered to the internal order
    const BoxState st = state();
    const int c = st.cur;
    std::vector<int32_t> tag(n);
    check_cuda(cudaMemcpy(tag.data(), desc.tag[c], sizeof(int) * n, cudaMemcpyDeviceToHost), "download");
    std::vector<double> col(n);
    for (int d = 0; d < 3; ++d) {
        if (x) {
            for (int i = 0; i < n; ++i) col[i] = x[3 * (tag[i] - 1) + d];
            check_cuda(cudaMemcpy(desc.x[c][d], col.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "upload");
        }
        if (v) {
            for (int i = 0; i < n; ++i) col[i] = v[3 * (tag[i] - 1) + d];
            check_cuda(cudaMemcpy(desc.v[c][d], col.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "upload");
        }
    }
}

// ---------------------------------------------------------------------------

Batch::Batch(std::vector<Box *> boxes, const StepConfig &c) : cfg(c), boxes_(std::move(boxes))
{
    if (boxes_.empty()) throw std::runtime_error("ARG: empty batch");
    cfg.uniform_types = 1;
    for (Box *b : boxes_) cfg.uniform_types &= b->desc.ntype == 1;
    cfg.half = cfg.style == 0 && !cfg.wall_coupling && cfg.half_enabled;
    check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    const int nb = (int)boxes_.size();
    d_boxes = batch_alloc<BoxDesc>(nb, stream_);
    std::vector<BoxDesc> h(nb);
    for (int b = 0; b < nb; ++b) {
        h[b] = boxes_[b]->desc;
        // the reduced list serves the pair-once passes only (the wall fix reads the full list)
        h[b].list_reduce = cfg.half && !cfg.wall && !h[b].wall_fix && !h[b].ab_mobile_bit &&
                           h[b].rn2_list < h[b].rc2_tail;
    }
    check_cuda(cudaMemcpyAsync(d_boxes, h.data(), sizeof(BoxDesc) * nb, cudaMemcpyHostToDevice, stream_), "boxes");
    d_done = batch_alloc<int>(4, stream_);
    check_cuda(cudaMemsetAsync(d_done, 0, sizeof(int) * 4, stream_), "done");
    d_thermo = batch_alloc<double>((size_t)kPartialStride * nb, stream_);
    d_states = batch_alloc<BoxState>(nb, stream_);
    build_units();  // synchronises the stream: h, the units and the counters are in place
    init_rebuild_shapes();  // occupancy queries stay out of the captures
    capture(0);
    capture(1);
}

Batch::~Batch()
{
    for (int k = 0; k < 2; ++k) {
        if (graph_[k]) cudaGraphExecDestroy(graph_[k]);
        if (graph_src_[k]) cudaGraphDestroy(graph_src_[k]);
    }
    // stream-ordered: after every kernel this batch queued; the stream is released once its
    // work is done
    for (Unit *u : unit_allocs_) cudaFreeAsync(u, stream_);
    for (void *p : {(void *)d_boxes, (void *)d_done, (void *)d_thermo, (void *)d_states})
        if (p) cudaFreeAsync(p, stream_);
    if (h_stage_) cudaFreeHost(h_stage_);
    for (auto &e : ev_stage_)
        if (e) cudaEventDestroy(e);
    if (stream_) cudaStreamDestroy(stream_);
}

// units of the boxes `which` (indices into the batch); device arrays appended to allocs
static BatchUnits make_units(const std::vector<Box *> &boxes, const std::vector<int> &which, int nbox,
                             std::vector<Unit *> &allocs, cudaStream_t s)
{
    std::vector<Unit> loc, all, cls, bins, scls, sgh, sbin;
    for (int b : which) {
        const BoxDesc &B = boxes[b]->desc;
        auto chunk = [&](std::vector<Unit> &v, int n, int step) {
            for (int s = 0; s < n; s += step) v.push_back({b, s, std::min(n, s + step)});
        };
        chunk(loc, B.nlocal, kUnit);
        chunk(all, B.nlocal + B.ghost_cap, kUnit);
        chunk(cls, 2 * B.nbin, 256);
        chunk(bins, B.nbin, 256);
        chunk(scls, 2 * B.nbin, kScanChunk);
        chunk(sgh, B.nlocal + 1, kScanChunk);
        chunk(sbin, B.nbin, kScanChunk);
    }
    auto up = [&](const std::vector<Unit> &v) {
        Unit *d = batch_alloc<Unit>(v.size(), s);
        if (!v.empty())
            check_cuda(cudaMemcpyAsync(d, v.data(), sizeof(Unit) * v.size(), cudaMemcpyHostToDevice, s), "units");
        allocs.push_back(d);
        return UnitList{d, (int)v.size()};
    };
    BatchUnits u;
    u.local = up(loc);
    u.all = up(all);
    u.cls = up(cls);
    u.bins = up(bins);
    u.scan_cls = up(scls);
    u.scan_ghost = up(sgh);
    u.scan_bin = up(sbin);
    u.nbox = nbox;  // box-indexed kernels (scan tops, build counters) see every box of the batch
    check_cuda(cudaStreamSynchronize(s), "units");  // the host vectors above are the copies' sources
    return u;
}

void Batch::build_units()
{
    std::vector<int> every(boxes_.size());
    for (size_t b = 0; b < boxes_.size(); ++b) every[b] = (int)b;
    units = make_units(boxes_, every, (int)boxes_.size(), unit_allocs_, stream_);
}

void Batch::capture(int ev)
{
    Range r("mdpd::capture");
    cudaGraph_t g;
    check_cuda(cudaGraphCreate(&g, 0), "graph create");
    cudaGraphConditionalHandle h;
    check_cuda(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault), "conditional handle");
    check_cuda(cudaStreamBeginCaptureToGraph(stream_, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
               "capture");
    launch_integrate(stream_, d_boxes, units, cfg, d_done, h, 1);
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    check_cuda(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, &cg, &deps, &nd), "capture info");
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t cn;
    check_cuda(cudaGraphAddNode(&cn, cg, deps, nd, &p), "conditional node");
    cudaGraph_t body = p.conditional.phGraph_out[0];
    check_cuda(cudaStreamUpdateCaptureDependencies(stream_, &cn, 1, cudaStreamSetCaptureDependencies), "deps");
    cudaStream_t s2;
    check_cuda(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking), "stream");
    check_cuda(cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
               "capture body");
    launch_rebuild(s2, d_boxes, units, cfg, d_done);
    cudaGraph_t tmp;
    check_cuda(cudaStreamEndCapture(s2, &tmp), "end body");
    cudaStreamDestroy(s2);
    if (cfg.style == 0) launch_density(stream_, d_boxes, units, cfg);
    launch_force(stream_, d_boxes, units, cfg, ev, 1);
    if (cfg.aboundary) launch_aboundary_meso(stream_, d_boxes, units);  // end of step, before output
    if (ev) launch_thermo(stream_, d_boxes, units, d_thermo, d_done + 2);
    check_cuda(cudaStreamEndCapture(stream_, &tmp), "end capture");
    check_cuda(cudaGraphInstantiate(&graph_[ev], g, 0), "instantiate");
    graph_src_[ev] = g;
}

void Batch::setup()
{
    Range r("mdpd::setup");
    launch_force_rebuild_flag(stream_, d_boxes, units.nbox, 1);
    launch_rebuild(stream_, d_boxes, units, cfg, d_done);
    if (cfg.style == 0) launch_density(stream_, d_boxes, units, cfg);
    launch_force(stream_, d_boxes, units, cfg, 1, 0);
    launch_force_rebuild_flag(stream_, d_boxes, units.nbox, 0);
    check_cuda(cudaGetLastError(), "setup launch");
    check_cuda(cudaStreamSynchronize(stream_), "setup");
}

__global__ void k_set_rebuild(BoxDesc *boxes, const int *which, int nwhich, int nbox)
{
    for (int b = threadIdx.x; b < nbox; b += blockDim.x) boxes[b].st->rebuild = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < nwhich; k += blockDim.x) {
        boxes[which[k]].st->rebuild = 1;
        boxes[which[k]].st->ago = 0;
    }
}

void Batch::setup_boxes(const std::vector<int> &which)
{
    Range r("mdpd::setup");
    if (which.empty()) return;
    int *d = batch_alloc<int>(which.size(), stream_);
    check_cuda(cudaMemcpyAsync(d, which.data(), sizeof(int) * which.size(), cudaMemcpyHostToDevice, stream_),
               "setup boxes");
    k_set_rebuild<<<1, 256, 0, stream_>>>(d_boxes, d, (int)which.size(), units.nbox);
    // the passes visit the new boxes only (the others keep their state and forces)
    std::vector<Unit *> allocs;
    const BatchUnits su = make_units(boxes_, which, units.nbox, allocs, stream_);
    launch_rebuild(stream_, d_boxes, su, cfg, d_done);
    if (cfg.style == 0) launch_density(stream_, d_boxes, su, cfg);
    launch_force(stream_, d_boxes, su, cfg, 1, 0);
    launch_force_rebuild_flag(stream_, d_boxes, units.nbox, 0);
    check_cuda(cudaFreeAsync(d, stream_), "setup boxes");
    for (Unit *a : allocs) cudaFreeAsync(a, stream_);
    check_cuda(cudaGetLastError(), "setup launch");
    check_cuda(cudaStreamSynchronize(stream_), "setup");
}

void Batch::reconfigure(const StepConfig &c)
{
    check_cuda(cudaStreamSynchronize(stream_), "reconfigure");
    for (int k = 0; k < 2; ++k) {
        if (graph_[k]) cudaGraphExecDestroy(graph_[k]);
        if (graph_src_[k]) cudaGraphDestroy(graph_src_[k]);
        graph_[k] = nullptr;
        graph_src_[k] = nullptr;
    }
    const int uni = cfg.uniform_types, half = cfg.half;
    cfg = c;
    cfg.uniform_types = uni;
    cfg.half = half;
    capture(0);
    capture(1);
}

void Batch::run(long long nsteps, bool sync, bool ev_last)
{
    Range r("mdpd::run");
    for (long long k = 0; k < nsteps; ++k)
        check_cuda(cudaGraphLaunch(graph_[ev_last && k == nsteps - 1 ? 1 : 0], stream_), "graph launch");
    if (sync) check_cuda(cudaStreamSynchronize(stream_), "run");
}

void Batch::step_ev() { check_cuda(cudaGraphLaunch(graph_[1], stream_), "graph launch"); }

long long Batch::rebuild_steps()
{
    int h[4];
    check_cuda(cudaMemcpy(h, d_done, sizeof(h), cudaMemcpyDeviceToHost), "counters");
    return h[3];
}

double Batch::time_pair_passes(int reps)
{
    Range r("mdpd::time_pair_passes");
    cudaEvent_t e0, e1;
    check_cuda(cudaEventCreate(&e0), "event");
    check_cuda(cudaEventCreate(&e1), "event");
    auto once = [&] {
        if (cfg.style == 0) launch_density(stream_, d_boxes, units, cfg);
        launch_force(stream_, d_boxes, units, cfg, 0, 0);
    };
    once();
    check_cuda(cudaEventRecord(e0, stream_), "event");
    for (int k = 0; k < reps; ++k) once();
    check_cuda(cudaEventRecord(e1, stream_), "event");
    check_cuda(cudaEventSynchronize(e1), "time pair passes");
    float t = 0;
    check_cuda(cudaEventElapsedTime(&t, e0, e1), "event");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_cuda(cudaGetLastError(), "time pair passes");
    return t / reps;
}

void Batch::profile(long long nsteps, double out[5])
{
    cudaEvent_t ev[5];
    for (auto &e : ev) check_cuda(cudaEventCreate(&e), "event");
    double acc[4] = {0, 0, 0, 0};
    const long long r0 = rebuild_steps();
    for (long long k = 0; k < nsteps; ++k) {
        cudaEventRecord(ev[0], stream_);
        {
            Range r("integrate");
            launch_integrate(stream_, d_boxes, units, cfg, d_done, cudaGraphConditionalHandle{}, 0);
        }
        cudaEventRecord(ev[1], stream_);
        {
            Range r("rebuild");
            launch_rebuild(stream_, d_boxes, units, cfg, d_done);  // kernels skip boxes not rebuilding
        }
        cudaEventRecord(ev[2], stream_);
        if (cfg.style == 0) {
            Range r("density");
            launch_density(stream_, d_boxes, units, cfg);
        }
        cudaEventRecord(ev[3], stream_);
        {
            Range r("force");
            launch_force(stream_, d_boxes, units, cfg, 0, 1);
            if (cfg.aboundary) launch_aboundary_meso(stream_, d_boxes, units);
        }
        cudaEventRecord(ev[4], stream_);
        check_cuda(cudaEventSynchronize(ev[4]), "profile");
        for (int q = 0; q < 4; ++q) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
            acc[q] += t;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (int q = 0; q < 4; ++q) out[q] = acc[q] / (double)nsteps;
    out[4] = (double)(rebuild_steps() - r0);
}

void Batch::thermo(std::vector<Thermo> &out)
{
    Range r("mdpd::thermo");
    launch_thermo(stream_, d_boxes, units, d_thermo, d_done + 2);
    check_cuda(cudaGetLastError(), "thermo launch");
    const int nb = (int)boxes_.size();
    std::vector<double> h((size_t)nb * kPartialStride);
    check_cuda(cudaMemcpyAsync(h.data(), d_thermo, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream_),
               "thermo download");
    check_cuda(cudaStreamSynchronize(stream_), "thermo");
    std::vector<BoxState> sts;
    read_states(sts);
    to_thermo(h.data(), sts.data(), out);
}

// every box's thermo from its reduced partials (kPartialStride doubles per box) and its scalars
void Batch::to_thermo(const double *h, const BoxState *sts, std::vector<Thermo> &out) const
{
    const int nb = (int)boxes_.size();
    out.resize(nb);
    for (int b = 0; b < nb; ++b) {
        const Box &bx = *boxes_[b];
        const BoxState &st = sts[b];
        Thermo &t = out[b];
        const double *q = &h[(size_t)b * kPartialStride];
        t.step = st.step;
        t.nbuild = st.nbuild;
        t.status = st.status;
        t.ke_all = q[0];
        for (int k = 0; k < 6; ++k) t.virial[k] = q[1 + k];
        t.pe = q[7];
        t.mom[0] = q[8], t.mom[1] = q[9], t.mom[2] = q[10];
        t.ke_group = q[11];
        for (int k = 0; k < 6; ++k) t.ke_tensor[k] = q[12 + k];
        t.n = bx.n;
        t.n_group = bx.n_group;
        // compute temp (all atoms, dof = 3N - 3) and pressure (compute_pressure_meso.cu:121-150)
        const double dof = 3.0 * t.n - 3.0;
        t.temp = dof > 0 ? t.ke_all / dof : 0.0;
        const double vol = bx.desc.prd[0] * bx.desc.prd[1] * bx.desc.prd[2];
        t.press = (dof * t.temp + t.virial[0] + t.virial[1] + t.virial[2]) / 3.0 / vol;
        // pressure tensor (compute pressure with keyword ke+virial, per component)
        for (int k = 0; k < 6; ++k) t.ptensor[k] = (t.ke_tensor[k] + t.virial[k]) / vol;
        t.surface_tension = 0.5 * bx.desc.prd[0] * (t.ptensor[0] - 0.5 * (t.ptensor[1] + t.ptensor[2]));
    }
}

void Batch::run_thermo(long long nsteps, const std::function<void(long long, const std::vector<Thermo> &)> &sink)
{
    Range r("mdpd::run_thermo");
    const int nb = (int)boxes_.size();
    const size_t part_bytes = sizeof(double) * kPartialStride * nb, st_bytes = sizeof(BoxState) * nb;
    if (!h_stage_) {
        check_cuda(cudaHostAlloc(&h_stage_, 2 * (part_bytes + st_bytes), cudaHostAllocDefault), "thermo staging");
        for (auto &e : ev_stage_) check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    }
    auto part = [&](int slot) { return reinterpret_cast<double *>(h_stage_ + slot * (part_bytes + st_bytes)); };
    auto states = [&](int slot) {
        return reinterpret_cast<BoxState *>(h_stage_ + slot * (part_bytes + st_bytes) + part_bytes);
    };
    std::vector<Thermo> t;
    for (long long k = 0; k <= nsteps; ++k) {
        if (k < nsteps) {  // step k and its thermo, queued
            const int slot = (int)(k & 1);
            // the step graph with energy and virial ends with the thermo reduction into d_thermo
            check_cuda(cudaGraphLaunch(graph_[1], stream_), "graph launch");
            launch_gather_states(stream_, d_boxes, nb, d_states);
            check_cuda(cudaGetLastError(), "thermo launch");
            check_cuda(cudaMemcpyAsync(part(slot), d_thermo, part_bytes, cudaMemcpyDeviceToHost, stream_), "thermo");
            check_cuda(cudaMemcpyAsync(states(slot), d_states, st_bytes, cudaMemcpyDeviceToHost, stream_), "states");
            check_cuda(cudaEventRecord(ev_stage_[slot], stream_), "event");
        }
        if (k >= 1) {  // step k - 1's results, while step k runs
            const int slot = (int)((k - 1) & 1);
            check_cuda(cudaEventSynchronize(ev_stage_[slot]), "thermo");
            to_thermo(part(slot), states(slot), t);
            sink(k - 1, t);
        }
    }
}

size_t Batch::thermo_bytes_per_step() const
{
    return (sizeof(double) * kPartialStride + sizeof(BoxState)) * boxes_.size();
}

void Batch::download_all(double *const *x, double *const *v)
{
    Range r("mdpd::download_all");
    size_t nmax = 0;
    for (const Box *b : boxes_) nmax = std::max(nmax, (size_t)b->n);
    if (nmax == 0) return;
    // one scratch of the largest box, reused box after box: the stream runs each box's gather
    // after the previous box's copies have read the scratch, so nothing waits on the host
    // until the end
    double *d = batch_alloc<double>(6 * nmax, stream_);
    for (size_t k = 0; k < boxes_.size(); ++k) {
        const Box *b = boxes_[k];
        const size_t n3 = 3 * (size_t)b->n;
        launch_gather_by_tag(stream_, state_buffers(b->desc), b->desc.st, b->n, d, d + n3);
        check_cuda(cudaGetLastError(), "download gather");
        if (x[k]) check_cuda(cudaMemcpyAsync(x[k], d, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream_), "download");
        if (v[k]) check_cuda(cudaMemcpyAsync(v[k], d + n3, sizeof(double) * n3, cudaMemcpyDeviceToHost, stream_), "download");
    }
    check_cuda(cudaFreeAsync(d, stream_), "download scratch");
    check_cuda(cudaStreamSynchronize(stream_), "download");
}

void Batch::read_states(std::vector<BoxState> &out)
{
    const int nb = (int)boxes_.size();
    out.resize(nb);
    launch_gather_states(stream_, d_boxes, nb, d_states);
    check_cuda(cudaGetLastError(), "states launch");
    check_cuda(cudaMemcpyAsync(out.data(), d_states, sizeof(BoxState) * nb, cudaMemcpyDeviceToHost, stream_),
               "states download");
    check_cuda(cudaStreamSynchronize(stream_), "states");
}

// names of the set bits of a box status word
std::string status_text(int bits)
{
    static const char *names[] = {"neighbour list overflow", "ghost capacity overflow", "bin/bucket overflow",
                                  "non-finite force", "particle lost", "compact list overflow",
                                  "index out of range (index-check build)"};
    std::string t;
    for (int k = 0; k < 7; ++k)
        if (bits & (1 << k)) t += (t.empty() ? "" : ", ") + std::string(names[k]);
    return t;
}

int Batch::status(std::string &msg)
{
    int all = 0;
    std::vector<BoxState> sts;
    read_states(sts);
    for (size_t b = 0; b < boxes_.size(); ++b) {
        const BoxState &st = sts[b];
        if (st.status) {
            all |= st.status;
            msg += "box " + std::to_string(b) + ": status " + std::to_string(st.status) + " (" +
                   status_text(st.status) + "); ";
        }
    }
    return all;
}

}  // namespace mdpd
