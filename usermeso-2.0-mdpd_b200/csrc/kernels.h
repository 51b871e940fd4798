// Host-side launchers of the device kernels.  Every launcher takes the device box table
// and a device list of work units; grids are persistent (a multiple of the SM count).
#pragma once

#include "mdpd_dev.cuh"

namespace mdpd {

struct UnitList {
    const Unit *d = nullptr;  // device array
    int n = 0;
};

// units of one batch, by domain (all boxes concatenated)
struct BatchUnits {
    UnitList local;      // [0,nlocal) in chunks of kUnit, 32-aligned
    UnitList all;        // [0,nlocal+ghost_cap) in chunks of kUnit
    UnitList cls;        // [0,2*nbin) in chunks of 256 buckets
    UnitList bins;       // [0,nbin) in chunks of 256 bins
    UnitList scan_cls;   // [0,2*nbin) in chunks of kScanChunk
    UnitList scan_ghost; // [0,nlocal+1)
    UnitList scan_bin;   // [0,nbin)
    int nbox = 0;
};

constexpr int kScanChunk = 2048;

struct StepConfig {
    int tpp_density = 1;   // threads per particle in the density pass
    int tpp_force = 1;     // threads per particle in the force pass
    int exact_rng = 0;     // FP64 bit-exact gaussian
    int wall = 0;          // aboundary bounce-back in the integrate pass
    int wall_coupling = 0; // phi-dependent gamma/sigma in the force pass
    int style = 0;         // 0 mdpd, 1 dpd
    int uniform_types = 0; // every box has one atom type: constant coefficient index
    int half = 0;          // mdpd without wall coupling: each pair evaluated once (k_pair.cu)
    int half_enabled = 1;  // allow the half-list passes (set per batch from the boxes)
    int gather = 6;        // pair-once density pass: neighbour positions in flight per lane (4, 6, 8)
    int stage_rows = 1;    // pair-once force pass: each warp's compact rows staged in shared memory
                           // (0: the pair loop reads its entries from the table)
    int aboundary = 0;     // fix aboundary/meso at the end of each step
    int sms = 148;
};

// scratch counter words used for last-block detection (device)
struct Counters {
    int *integrate;
    int *rebuild_last;
};

void launch_integrate(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c,
                      int *done, cudaGraphConditionalHandle cond, int use_cond);
void launch_force_rebuild_flag(cudaStream_t s, BoxDesc *boxes, int nbox, int value);
void launch_rebuild(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c,
                    int *done);
// the rebuild passes' grid sizes from the occupancy API: call once before any stream capture
void init_rebuild_shapes();
void launch_density(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c);
void launch_force(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int ev,
                  int kick);
void launch_aboundary_meso(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u);
void launch_density_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c);
void launch_force_half(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, const StepConfig &c, int ev, int kick);
// AoS x[3n] (and v[3n], or zero when null) -> components x[d], xh[d], v[d]; tags 1..n, type 1
// and mask 1 into the arrays given (null: left as uploaded)
void launch_load_state(cudaStream_t s, const double *xa, const double *va, int n, double *const x[3],
                       double *const xh[3], double *const v[3], int *tag, int *type, int *mask);
// Morton rank of every bin of an mbin[0] x mbin[1] x mbin[2] grid (bin x + mx (y + my z))
void launch_bin_ranks(cudaStream_t s, const int mbin[3], int *rank);
// copies of every box's BoxState into out[nbox]
void launch_gather_states(cudaStream_t s, const BoxDesc *boxes, int nbox, BoxState *out);
// both buffers of a box's double-buffered x, v (components) and tags
struct StateBuffers {
    const double *x[2][3], *v[2][3];
    const int *tag[2];
};
// x, v of the live buffer (st->cur, read on the device), internal order -> xo[3n], vo[3n] in
// tag order (tags 1..n)
void launch_gather_by_tag(cudaStream_t s, const StateBuffers &b, const BoxState *st, int n, double *xo, double *vo);
void launch_thermo(cudaStream_t s, BoxDesc *boxes, const BatchUnits &u, double *out, int *done);
void launch_density_profile(cudaStream_t s, const BoxDesc *boxes, int box, const Unit *units,
                            int nunits, int dim, int groupbit, double lo, double inv, int nbin,
                            unsigned long long *counts);
// test hooks: the pair RNG on explicit signatures
void launch_gaussian(cudaStream_t s, const uint32_t *si, const uint32_t *sj, double *exact,
                     float *fast, int n);

}  // namespace mdpd
