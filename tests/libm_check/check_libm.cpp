// Host check of the product's exp/log/sin/cos (anionpy_b200/csrc/ionp_libm.cuh,
// compiled here for the CPU) against the host C library, the oracle of the
// transcendental ufuncs. Every result must have the same bits, NaNs included.
//   check_libm f32 <stride>   every stride-th float32 bit pattern, exp/log/sin/cos
//   check_libm f64 <count>    count seeded float64 arguments per function,
//                             drawn from ranges that reach every code path
// Prints one line per function: "<name> n=<checked> diff=<mismatches>".
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>
#include "ionp_libm.cuh"

using namespace ionp::lm;

static uint64_t next(uint64_t s[2]) {
    uint64_t a = s[0];
    const uint64_t b = s[1];
    s[0] = b;
    a ^= a << 23;
    s[1] = a ^ b ^ (a >> 17) ^ (b >> 26);
    return s[1] + b;
}

template <class F> static void run(const char* name, uint64_t n, int nt, F body) {
    std::atomic<uint64_t> diff{0}, done{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t]() {
            uint64_t d = 0, c = 0;
            body(t, nt, &d, &c);
            diff += d;
            done += c;
        });
    for (auto& x : th) x.join();
    printf("%s n=%llu diff=%llu\n", name, (unsigned long long)done.load(), (unsigned long long)diff.load());
}

static double draw(uint64_t u, int cls, int fn) {
    const double U = (double)(u >> 11) * 0x1p-53;
    switch (cls) {
        case 0: return dfrom(u);                                            // any bits
        case 1: return dfrom((u & 0x800FFFFFFFFFFFFFull) | ((uint64_t)(900 + (u >> 52) % 250) << 52));
        case 2: return fn == 0 ? (U - 0.5) * 1500.0 : fn == 1 ? 1e6 * (1.0 - U) : (U - 0.5) * 200.0;
        case 3: return fn == 0 ? -708.0 - 37.0 * U : fn == 1 ? 0.9 + 0.2 * U : (U - 0.5) * 4.8;
        case 4: return fn == 0 ? 705.0 + 5.0 * U : fn == 1 ? dfrom(u & 0x000FFFFFFFFFFFFFull)
                                                       : dfrom((u & 0x800FFFFFFFFFFFFFull) | ((uint64_t)(1049 + (u >> 52) % 980) << 52));
        default: return (U - 0.5) * 2.0;
    }
}

int main(int argc, char** argv) {
    const int nt = (int)std::thread::hardware_concurrency();
    const bool f32 = argc > 1 && !strcmp(argv[1], "f32");
    const uint64_t arg = argc > 2 ? strtoull(argv[2], nullptr, 10) : 1;
    if (f32) {
        const uint64_t stride = arg ? arg : 1;
        const char* names[4] = {"exp32", "log32", "sin32", "cos32"};
        for (int fn = 0; fn < 4; fn++)
            run(names[fn], 0, nt, [&](int t, int T, uint64_t* d, uint64_t* c) {
                for (uint64_t u = (uint64_t)t * stride; u <= 0xFFFFFFFFull; u += (uint64_t)T * stride) {
                    const float x = ffrom((uint32_t)u);
                    const float m = fn == 0 ? exp32(x) : fn == 1 ? log32(x) : fn == 2 ? sin32(x) : cos32(x);
                    const float g = fn == 0 ? expf(x) : fn == 1 ? logf(x) : fn == 2 ? sinf(x) : cosf(x);
                    ++*c;
                    if (fbits(m) != fbits(g)) ++*d;
                }
            });
    } else {
        const char* names[4] = {"exp64", "log64", "sin64", "cos64"};
        for (int fn = 0; fn < 4; fn++)
            run(names[fn], 0, nt, [&](int t, int T, uint64_t* d, uint64_t* c) {
                uint64_t st[2] = {0x9E3779B97F4A7C15ull * (uint64_t)(t + 1 + 64 * fn), 0xD1B54A32D192ED03ull};
                for (uint64_t i = (uint64_t)t; i < arg; i += (uint64_t)T) {
                    const double x = draw(next(st), (int)(i % 6), fn < 3 ? fn : 2);   // cos: sin's ranges
                    const double m = fn == 0 ? exp64(x) : fn == 1 ? log64(x) : fn == 2 ? sin64(x) : cos64(x);
                    const double g = fn == 0 ? exp(x) : fn == 1 ? log(x) : fn == 2 ? sin(x) : cos(x);
                    ++*c;
                    if (dbits(m) != dbits(g)) ++*d;
                }
            });
    }
    return 0;
}
