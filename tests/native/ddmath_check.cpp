// Host check of setsm_b200/csrc/vll_ddmath.cuh against the C library: per
// function, the arguments whose result differs from the library's.  Prints
// "count <name> <tried> <differing>" per function and, for the first
// differing arguments, "diff <name> <x> [<y>] <ours> <library>" in hex floats
// (tests/test_ddmath.py checks those against 300-bit arithmetic).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "vll_ddmath.cuh"

using namespace vll::ddm;

int main(int argc, char **argv) {
    const long n = argc > 1 ? atol(argv[1]) : 200000;
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> u(0.0, 1.0);
    auto logu = [&](double lo, double hi) { return lo * std::pow(hi / lo, u(rng)); };
    auto sgn = [&]() { return u(rng) < 0.5 ? -1.0 : 1.0; };
    long bad[7] = {0}, cnt[7] = {0};
    const char *names[7] = {"sin", "cos", "tan", "atan", "atan2", "exp", "acos"};
    auto note = [&](int f, double ours, double lib, double x, double y, bool two) {
        cnt[f]++;
        if (ours == lib) return;
        if (bad[f]++ < 20) {
            if (two) printf("diff %s %a %a %a %a\n", names[f], x, y, ours, lib);
            else printf("diff %s %a %a %a\n", names[f], x, ours, lib);
        }
    };
    for (long i = 0; i < n; ++i) {
        const double a = (u(rng) * 2 - 1) * 26.0;            // the projection's angle range
        const double b = sgn() * logu(1e-9, 3.0);
        for (double x : {a, b}) {
            note(0, sin_cr(x), std::sin(x), x, 0, false);
            note(1, cos_cr(x), std::cos(x), x, 0, false);
            note(2, tan_cr(x), std::tan(x), x, 0, false);
        }
        const double t = sgn() * logu(1e-8, 1e8);
        note(3, atan_cr(t), std::atan(t), t, 0, false);
        const double y = sgn() * logu(1e-3, 1e7), xx = sgn() * logu(1e-3, 1e7);
        note(4, atan2_cr(y, xx), std::atan2(y, xx), y, xx, true);
        const double e = u(rng) < 0.5 ? (u(rng) * 2 - 1) * 3.0 : (u(rng) * 2 - 1) * 700.0;
        note(5, exp_cr(e), std::exp(e), e, 0, false);
        const double ac = u(rng) < 0.5 ? (u(rng) * 2 - 1) : sgn() * (1.0 - logu(1e-12, 1e-2));
        note(6, acos_cr(ac), std::acos(ac), ac, 0, false);
    }
    for (int f = 0; f < 7; ++f) printf("count %s %ld %ld\n", names[f], cnt[f], bad[f]);
    return 0;
}
