// Placement of independent boxes or jobs on the GPUs of a node (host only, no device work).
//
// The reference runs an ensemble of independent cases by splitting MPI_COMM_WORLD into groups of
// case_size ranks, each group reading one line of an argument file (main_ensemble,
// src/main.cpp:49-117): case k goes to ranks [k case_size, (k + 1) case_size) whatever its size.
// Here a case is one box and a rank is one GPU, and boxes differ in size by two orders of
// magnitude (2k-200k particles in a batch, 5k-2M in served jobs), so the placement balances
// their work instead of their count, under each device's HBM budget:
//   items in decreasing work (particles times steps; ties by index), each to the device with the
//   least work placed so far among those whose bytes still fit (ties: the lower device).
// This is the longest-processing-time rule: within 4/3 of the best balance for any item set, and
// within a few per cent for hundreds of uneven boxes.  The result depends only on the inputs, so
// every rank computes the same placement and takes its own share without exchanging anything.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "../../include/mdpd.h"

extern "C" int mdpd_place(const mdpd_box_spec *specs, const int64_t *steps, int32_t nitem, int32_t ndev,
                          const uint64_t *budget_bytes, int32_t *device_of, double *work_per_device)
{
    if (!specs || nitem < 0 || ndev <= 0 || !budget_bytes || !device_of) return MDPD_ERR_ARG;
    std::vector<double> work(nitem);
    std::vector<uint64_t> bytes(nitem);
    for (int32_t i = 0; i < nitem; ++i) {
        if (steps && steps[i] < 0) return MDPD_ERR_ARG;
        if (mdpd_box_bytes(&specs[i], &bytes[i]) != MDPD_OK) return MDPD_ERR_ARG;
        work[i] = (double)specs[i].n * (double)(steps ? steps[i] : 1);
    }
    std::vector<int32_t> order(nitem);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return work[a] > work[b]; });
    std::vector<double> load(ndev, 0.0);
    std::vector<uint64_t> used(ndev, 0);
    int rc = MDPD_OK;
    for (int32_t i : order) {
        int best = -1;
        for (int d = 0; d < ndev; ++d) {
            if (used[d] + bytes[i] > budget_bytes[d] || used[d] + bytes[i] < used[d]) continue;
            if (best < 0 || load[d] < load[best]) best = d;
        }
        device_of[i] = best;
        if (best < 0) {
            rc = MDPD_ERR_BUDGET;
            continue;
        }
        load[best] += work[i];
        used[best] += bytes[i];
    }
    if (work_per_device)
        for (int d = 0; d < ndev; ++d) work_per_device[d] = load[d];
    return rc;
}
