// Unit test of mdp::PerDeviceMemo (mdp_b200/csrc/device_cache.h): the launch
// set-up of a kernel (its shared-memory attribute and occupancy) runs once per
// (kernel, device), a second device gets its own set-up, a failed set-up is
// retried, and concurrent first calls run the set-up once.  Exit status 0 on
// success; prints the first failed check otherwise.
#include "device_cache.h"

#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

static int fails = 0;
#define CHECK(c)                                                      \
    do {                                                              \
        if (!(c)) {                                                   \
            std::printf("FAILED line %d: %s\n", __LINE__, #c);        \
            fails++;                                                  \
        }                                                             \
    } while (0)

static void kernel_a() {}
static void kernel_b() {}

int main()
{
    mdp::PerDeviceMemo memo;
    int calls[2] = {0, 0};
    auto setup_on = [&](int dev, int value) {
        return [&calls, dev, value](int *v) {
            calls[dev]++;
            *v = value;
            return 0;
        };
    };
    const void *ka = (const void *)&kernel_a, *kb = (const void *)&kernel_b;
    int v = 0;
    CHECK(memo.get(ka, 1024, 0, setup_on(0, 3), &v) == 0 && v == 3);
    CHECK(memo.get(ka, 1024, 0, setup_on(0, 99), &v) == 0 && v == 3);   // cached on device 0
    CHECK(calls[0] == 1);
    CHECK(memo.get(ka, 1024, 1, setup_on(1, 2), &v) == 0 && v == 2);    // device 1: its own set-up
    CHECK(calls[1] == 1);
    CHECK(memo.get(ka, 2048, 1, setup_on(1, 1), &v) == 0 && v == 1);    // another tag (shared size)
    CHECK(calls[1] == 2);
    CHECK(memo.get(kb, 1024, 0, setup_on(0, 5), &v) == 0 && v == 5);    // another kernel
    CHECK(calls[0] == 2);
    CHECK(memo.size() == 4);

    // a failed set-up caches nothing and is retried
    int tries = 0;
    auto failing = [&tries](int *v) { tries++; *v = 7; return tries < 2 ? -1 : 0; };
    v = -1;
    CHECK(memo.get(kb, 1024, 1, failing, &v) == -1 && v == -1);
    CHECK(memo.get(kb, 1024, 1, failing, &v) == 0 && v == 7);
    CHECK(memo.get(kb, 1024, 1, failing, &v) == 0 && tries == 2);

    // first calls from many host threads at once: one set-up per device
    mdp::PerDeviceMemo memo2;
    std::atomic<int> setups{0};
    std::vector<std::thread> th;
    std::atomic<int> bad{0};
    for (int t = 0; t < 16; t++)
        th.emplace_back([&, t] {
            const int dev = t & 1;
            for (int rep = 0; rep < 200; rep++) {
                int out = 0;
                auto s = [&setups, dev](int *x) { setups++; *x = 10 + dev; return 0; };
                if (memo2.get(ka, 64, dev, s, &out) || out != 10 + dev) bad++;
            }
        });
    for (auto &x : th) x.join();
    CHECK(bad == 0);
    CHECK(setups == 2);
    if (fails == 0) std::printf("ok\n");
    return fails ? 1 : 0;
}
