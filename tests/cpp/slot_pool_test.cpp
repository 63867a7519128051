// CPU test of the multi-GPU dispatch policy (segalign_b200/csrc/sa_slot_pool.h)
// with a faked device count: a pool of n_dev x per_dev slots guarded by a
// mutex and condition variable, as sa_api.cu holds it, and n_threads callers
// that take a slot, hold it for a while and give it back.
// Checks: no slot is ever held twice; every device serves calls; a device
// takes a further slot only when no less-loaded device has a free slot; and
// the first n_dev concurrent callers land on n_dev different devices.
// Prints "ok" and the per-device call counts.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#include "sa_slot_pool.h"

struct Slot {
    int dev;
    std::atomic<int> holders{0};
};

int main(int argc, char** argv) {
    const int n_dev = argc > 1 ? atoi(argv[1]) : 4;
    const int per_dev = argc > 2 ? atoi(argv[2]) : 3;
    const int n_threads = argc > 3 ? atoi(argv[3]) : 16;
    const int calls = argc > 4 ? atoi(argv[4]) : 400;
    std::vector<Slot> slots(n_dev * per_dev);
    std::deque<Slot*> free_slots;
    // device-major order, as slots are created
    for (int d = 0; d < n_dev; ++d)
        for (int k = 0; k < per_dev; ++k) {
            slots[d * per_dev + k].dev = d;
            free_slots.push_back(&slots[d * per_dev + k]);
        }
    std::mutex mu;
    std::condition_variable cv;
    std::vector<int> busy(n_dev, 0), served(n_dev, 0);
    bool bad = false;
    auto take = [&]() {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !free_slots.empty(); });
        std::vector<int> dev(free_slots.size());
        for (size_t i = 0; i < dev.size(); ++i) dev[i] = free_slots[i]->dev;
        const size_t k = sa_pick_free_slot(dev, n_dev);
        Slot* s = free_slots[k];
        free_slots.erase(free_slots.begin() + (long)k);
        ++busy[s->dev];
        ++served[s->dev];
        // balance: the chosen device was not busier than a device with a free slot
        for (int d = 0; d < n_dev; ++d)
            if (busy[d] < busy[s->dev] - 1 && busy[d] < per_dev) bad = true;
        return s;
    };
    auto give = [&](Slot* s) {
        {
            std::lock_guard<std::mutex> lk(mu);
            --busy[s->dev];
            free_slots.push_back(s);
        }
        cv.notify_all();
    };
    // first n_dev concurrent callers: distinct devices
    {
        std::vector<Slot*> first;
        for (int i = 0; i < n_dev; ++i) first.push_back(take());
        std::vector<int> seen(n_dev, 0);
        for (Slot* s : first) seen[s->dev]++;
        for (int d = 0; d < n_dev; ++d)
            if (seen[d] != 1) {
                printf("FAIL: first %d callers not on distinct devices\n", n_dev);
                return 1;
            }
        for (Slot* s : first) give(s);
    }
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < n_threads; ++t)
        th.emplace_back([&, t]() {
            std::mt19937 rng(t);
            while (next.fetch_add(1) < calls) {
                Slot* s = take();
                if (s->holders.fetch_add(1) != 0) bad = true;  // held twice
                std::this_thread::sleep_for(std::chrono::microseconds(50 + rng() % 200));
                s->holders.fetch_sub(1);
                give(s);
            }
        });
    for (auto& x : th) x.join();
    for (int d = 0; d < n_dev; ++d)
        if (served[d] == 0) bad = true;
    if (bad || (int)free_slots.size() != n_dev * per_dev) {
        printf("FAIL\n");
        return 1;
    }
    printf("ok");
    for (int d = 0; d < n_dev; ++d) printf(" %d", served[d]);
    printf("\n");
    return 0;
}
