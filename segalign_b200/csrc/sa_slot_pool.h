// sa_slot_pool.h — which free slot a SeedAndFilter call takes.
//
// The reference hands each call a whole GPU from a mutex/condition-variable
// pool of device ids (src/seed_filter.cu:667-674, released at :748-753), so
// concurrent calls spread over the GPUs one per device.  Here a GPU holds
// several slots (stream + workspace), and a call takes the first free slot,
// in pool order, of the device with the most free slots: k concurrent calls
// on G GPUs land on min(k, G) different devices before any device takes a
// second one.  Header-only and CUDA-free, so the policy is tested on the CPU.
#pragma once

#include <cstddef>
#include <vector>

// free_dev[i] = device of the i-th free slot (pool order); n_dev devices.
// Returns the index of the slot to take (free_dev must not be empty).
inline size_t sa_pick_free_slot(const std::vector<int>& free_dev, int n_dev) {
    std::vector<int> cnt(n_dev > 0 ? n_dev : 1, 0);
    for (int d : free_dev)
        if (d >= 0 && d < n_dev) ++cnt[d];
    size_t best = 0;
    for (size_t i = 1; i < free_dev.size(); ++i) {
        const int a = free_dev[i], b = free_dev[best];
        if (a >= 0 && a < n_dev && (b < 0 || b >= n_dev || cnt[a] > cnt[b])) best = i;
    }
    return best;
}
