// Pair-parallel batches over several GPUs (elas_b200_group_*).
//
// The reference has no multi-GPU code; its process() runs one pair on
// device 0 (src/Elas.h:70-83).  Stereo pairs are independent, so a batch
// spreads over devices with no exchange at all: a plan deals the pairs to
// the devices by estimated cost (largest first, each to the least-loaded
// device), and every device runs its share as one batch call on its own
// handle from its own host thread.  No peer memory is touched and no
// collective runs; the outputs equal single-pair runs bit for bit, because
// each pair runs the single-pair kernels on one device.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/elas_b200.h"

struct elas_group {
    std::vector<int> devices;
    std::vector<elas_handle*> handles;   // one per entry of `devices`
    std::string last_error;
};

namespace {

// Relative cost of a pair: the dense and support stages scale with the
// pixels times the disparity range, the rest with the pixels.
double pair_cost(int32_t w, int32_t h, int32_t dmax) {
    return double(w) * double(h) * (1.0 + double(dmax) / 128.0);
}

}  // namespace

extern "C" {

int elas_b200_group_plan(int n, const int32_t* dims, const int32_t* disp_max_per_pair, int32_t disp_max, int ndev,
                         int32_t* assign) {
    if (n < 0 || ndev < 1 || (n > 0 && (!dims || !assign))) return ELAS_ERR_INVALID_ARG;
    std::vector<int> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    std::vector<double> cost(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i)
        cost[size_t(i)] = pair_cost(dims[2 * i], dims[2 * i + 1], disp_max_per_pair ? disp_max_per_pair[i] : disp_max);
    // largest first; equal costs keep pair order, so the plan is deterministic
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[size_t(a)] > cost[size_t(b)]; });
    std::vector<double> load(static_cast<size_t>(ndev), 0.0);
    for (int i : order) {
        int best = 0;
        for (int d = 1; d < ndev; ++d)
            if (load[size_t(d)] < load[size_t(best)]) best = d;
        assign[i] = best;
        load[size_t(best)] += cost[size_t(i)];
    }
    return ELAS_OK;
}

int elas_b200_group_create(const elas_params* params, const int32_t* devices, int ndev, elas_group** out) {
    if (!out || !devices || ndev < 1) return ELAS_ERR_INVALID_ARG;
    *out = nullptr;
    elas_group* g = new elas_group();
    for (int k = 0; k < ndev; ++k) {
        elas_handle* h = nullptr;
        const int rc = elas_b200_create(params, devices[k], &h);
        if (rc != ELAS_OK) {
            for (elas_handle* x : g->handles) elas_b200_destroy(x);
            delete g;
            return rc;
        }
        g->devices.push_back(devices[k]);
        g->handles.push_back(h);
    }
    *out = g;
    return ELAS_OK;
}

int elas_b200_group_destroy(elas_group* g) {
    if (!g) return ELAS_ERR_INVALID_ARG;
    for (elas_handle* h : g->handles) elas_b200_destroy(h);
    delete g;
    return ELAS_OK;
}

int elas_b200_group_set_params(elas_group* g, const elas_params* params) {
    if (!g || !params) return ELAS_ERR_INVALID_ARG;
    for (elas_handle* h : g->handles) {
        const int rc = elas_b200_set_params(h, params);
        if (rc != ELAS_OK) {
            g->last_error = elas_b200_last_error(h);
            return rc;
        }
    }
    return ELAS_OK;
}

const char* elas_b200_group_last_error(const elas_group* g) { return g ? g->last_error.c_str() : ""; }

int elas_b200_group_process_batch(elas_group* g, int n, const uint8_t* const* lefts, const uint8_t* const* rights,
                                  float* const* disp_lefts, float* const* disp_rights, const int32_t* dims,
                                  const int32_t* disp_max_per_pair, int32_t* assign_out) {
    if (!g || n < 0 || (n > 0 && (!lefts || !rights || !disp_lefts || !disp_rights || !dims)))
        return ELAS_ERR_INVALID_ARG;
    if (n == 0) return ELAS_OK;
    const int ndev = int(g->handles.size());
    elas_params p;
    elas_b200_get_params(g->handles[0], &p);
    std::vector<int32_t> assign(static_cast<size_t>(n));
    int rc = elas_b200_group_plan(n, dims, disp_max_per_pair, p.disp_max, ndev, assign.data());
    if (rc != ELAS_OK) return rc;
    if (assign_out) std::memcpy(assign_out, assign.data(), size_t(n) * sizeof(int32_t));
    // each device's share as its own batch (pointer and size arrays gathered in pair order)
    struct Share {
        std::vector<const uint8_t*> l, r;
        std::vector<float*> d1, d2;
        std::vector<int32_t> dims, dmax;
        int rc = ELAS_OK;
    };
    std::vector<Share> share(static_cast<size_t>(ndev));
    for (int i = 0; i < n; ++i) {
        Share& s = share[size_t(assign[size_t(i)])];
        s.l.push_back(lefts[i]);
        s.r.push_back(rights[i]);
        s.d1.push_back(disp_lefts[i]);
        s.d2.push_back(disp_rights[i]);
        s.dims.push_back(dims[2 * i]);
        s.dims.push_back(dims[2 * i + 1]);
        s.dmax.push_back(disp_max_per_pair ? disp_max_per_pair[i] : p.disp_max);
    }
    std::vector<std::thread> workers;
    for (int d = 0; d < ndev; ++d) {
        Share& s = share[size_t(d)];
        if (s.l.empty()) continue;
        elas_handle* h = g->handles[size_t(d)];
        workers.emplace_back([&s, h] {
            s.rc = elas_b200_process_batch(h, int(s.l.size()), s.l.data(), s.r.data(), s.d1.data(), s.d2.data(),
                                           s.dims.data(), s.dmax.data(), nullptr);
        });
    }
    for (std::thread& t : workers) t.join();
    for (int d = 0; d < ndev; ++d)
        if (share[size_t(d)].rc != ELAS_OK) {
            g->last_error = "device " + std::to_string(g->devices[size_t(d)]) + ": " +
                            elas_b200_last_error(g->handles[size_t(d)]);
            return share[size_t(d)].rc;
        }
    return ELAS_OK;
}

}  // extern "C"
