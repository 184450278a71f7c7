// Host-side check of asg::div_by (astrosimgpu_b200/csrc/asg_device.cuh), the
// division by a run-time constant through its correctly rounded reciprocal
// with one FMA correction.  The engine relies on div_by(a, b, RN(1/b)) being
// bitwise the IEEE quotient a / b that the reference computes.  The host's
// fma is the correctly rounded fused multiply-add of IEEE 754, as the GPU's
// DFMA is, so the identity checked here is the identity the kernels rely on.
//
// Test infrastructure: built and run by tests/test_div_by.py.
//
//   div_by_check <random cases> <seed>
//
// prints one line per class of operands: "<class> <cases> <mismatches>".
//   random      a, b with random signs, exponents in [-960, 960] and
//               mantissas: the quotient and the remainder are normal, the
//               domain of Markstein's theorem
//   engine      b from the engine's divisors (ratio_ER_cyt, tau_IP3 spread,
//               C_m, Delta_T, tau_w, tau_rec, tau_fac of the shipped
//               configs), a of the magnitudes the model's numerators take
//               (1e-300 .. 1e6, both signs)
//   tiny_a      |a| below 2^-969 with a normal quotient: the remainder can be
//               subnormal (outside the theorem)
//   sub_q       subnormal quotients (outside the theorem)
//   huge        quotients and numerators near the overflow threshold
//   hard        mantissas of all ones, powers of two and near-powers of two
//   zero        a = +0 (and, separately, a = -0 in class neg_zero, whose IEEE
//               quotient is -0)
//   diff        div_diff_by(x, y, b, RN(1/b)) against IEEE (x - y) / b, where
//               x or y is a parameter of magnitude in [2^-906, 2^976] and the
//               other operand is anything finite: near-equal, equal, zero,
//               subnormal, or of any magnitude (|x - y| < 2^977)
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "asg_device.cuh"

namespace {

std::uint64_t bits(double x) {
    std::uint64_t u;
    std::memcpy(&u, &x, sizeof u);
    return u;
}

double from_bits(std::uint64_t u) {
    double x;
    std::memcpy(&x, &u, sizeof x);
    return x;
}

struct Rng {
    std::uint64_t s;
    std::uint64_t next() {  // splitmix64 sequence
        std::uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double unit() { return static_cast<double>(next() >> 11) * 0x1p-53; }
    // random sign, exponent in [lo, hi], random 52-bit mantissa
    double value(int lo, int hi) {
        const std::uint64_t r = next();
        const int e = lo + static_cast<int>(r % static_cast<std::uint64_t>(hi - lo + 1));
        const std::uint64_t mant = next() & ((1ULL << 52) - 1);
        const std::uint64_t sign = (r >> 63) << 63;
        return from_bits(sign | (static_cast<std::uint64_t>(e + 1023) << 52) | mant);
    }
};

struct Tally {
    const char* name;
    long long cases = 0, bad = 0;
    void check(double a, double b) {
        const double y = 1.0 / b;
        const double got = asg::div_by(a, b, y);
        const double want = a / b;
        ++cases;
        if (bits(got) != bits(want)) {
            if (bad < 3)
                std::fprintf(stderr, "%s: a=%a b=%a div_by=%a ieee=%a\n", name, a, b, got, want);
            ++bad;
        }
    }
    void print() const { std::printf("%s %lld %lld\n", name, cases, bad); }
};

}  // namespace

int main(int argc, char** argv) {
    const long long n = argc > 1 ? std::atoll(argv[1]) : 10000000LL;
    Rng rng{argc > 2 ? std::strtoull(argv[2], nullptr, 10) : 1ULL};

    Tally random{"random"};
    for (long long i = 0; i < n; ++i) {
        const double a = rng.value(-960, 960);
        const double b = rng.value(-60, 60);
        random.check(a, b);
    }

    // Divisors of the shipped configurations and their randomised spreads.
    const double divisors[] = {0.185, 1058.7589568400845, 1000.0, 200.0, 281.0, 250.0,
                               2.0,   1.0,   144.0, 600.0, 800.0, 1500.0, 50.0, 100.0, 3.0, 7.0};
    Tally engine{"engine"};
    for (long long i = 0; i < n / 4; ++i) {
        double b = divisors[rng.next() % (sizeof divisors / sizeof divisors[0])];
        if (rng.next() & 1) b *= 1.0 + 0.2 * (2.0 * rng.unit() - 1.0);  // per-cell spread
        const double a = rng.value(-996, 20);                           // ~1e-300 .. 1e6
        engine.check(a, b);
    }

    Tally tiny{"tiny_a"};
    for (long long i = 0; i < n / 20; ++i) {
        const double b = rng.value(-40, 0);                  // |b| < 2: normal quotient
        const double a = rng.value(-1020, -970);             // |a| < 2^-969
        if (std::fabs(a / b) >= 0x1p-1022) tiny.check(a, b);
    }

    Tally subq{"sub_q"};
    for (long long i = 0; i < n / 20; ++i) {
        const double b = rng.value(1, 60);
        const double a = from_bits((rng.next() & 0x800FFFFFFFFFFFFFULL) |
                                   (static_cast<std::uint64_t>(1 + rng.next() % 40) << 52));
        if (std::fabs(a / b) < 0x1p-1022 && a / b != 0.0) subq.check(a, b);
    }

    Tally huge{"huge"};
    for (long long i = 0; i < n / 20; ++i) {
        const double b = rng.value(-4, 4);
        const double a = rng.value(1015, 1023);
        huge.check(a, b);
    }

    Tally hard{"hard"};
    for (int eb = -20; eb <= 20; ++eb) {
        for (int ea = -20; ea <= 20; ++ea) {
            const double ones_a = std::ldexp(2.0 - 0x1p-52, ea), ones_b = std::ldexp(2.0 - 0x1p-52, eb);
            const double pa = std::ldexp(1.0, ea), pb = std::ldexp(1.0, eb);
            for (double a : {ones_a, pa, std::nextafter(pa, 0.0), std::nextafter(pa, 1e300), -ones_a})
                for (double b : {ones_b, pb, std::nextafter(pb, 0.0), std::nextafter(pb, 1e300)})
                    hard.check(a, b);
        }
    }
    for (long long i = 0; i < n / 20; ++i) {  // mantissas with long runs of ones/zeros
        const std::uint64_t run = (1ULL << (rng.next() % 52)) - 1;
        const double a = from_bits((static_cast<std::uint64_t>(1023 + rng.next() % 64) << 52) |
                                   ((rng.next() & 1) ? run : (~run & ((1ULL << 52) - 1))));
        const double b = from_bits((static_cast<std::uint64_t>(1023 - rng.next() % 64) << 52) |
                                   (rng.next() & ((1ULL << 52) - 1)));
        hard.check(a, b);
    }

    Tally zero{"zero"}, negzero{"neg_zero"};
    for (double b : divisors) {
        zero.check(0.0, b);
        negzero.check(-0.0, b);
    }

    // Divided differences with a parameter operand (div_diff_by).
    struct DiffTally : Tally {
        void check_diff(double x, double y, double b) {
            const double want = (x - y) / b;
            const double got = asg::div_diff_by(x, y, b, 1.0 / b);
            ++cases;
            if (bits(got) != bits(want)) {
                if (bad < 3)
                    std::fprintf(stderr, "%s: x=%a y=%a b=%a got=%a ieee=%a\n", name, x, y, b, got,
                                 want);
                ++bad;
            }
        }
    } diff;
    diff.name = "diff";
    for (long long i = 0; i < n / 4; ++i) {
        const double p = rng.value(-906, 975);
        double other;
        switch (rng.next() % 6) {
            case 0: other = p * (1.0 + std::ldexp(2.0 * rng.unit() - 1.0, -(int)(rng.next() % 50))); break;
            case 1: other = p; break;
            case 2: other = (rng.next() & 1) ? 0.0 : -0.0; break;
            case 3: other = from_bits(rng.next() & 0x800FFFFFFFFFFFFFULL); break;  // subnormal
            case 4: other = rng.value(-1022, 975); break;
            default: other = std::nextafter(p, (rng.next() & 1) ? 1e308 : -1e308); break;
        }
        double b = (rng.next() & 1) ? divisors[rng.next() % (sizeof divisors / sizeof divisors[0])]
                                    : std::fabs(rng.value(-46, 62));
        if (rng.next() & 1) b = -b;
        const bool param_first = rng.next() & 1;
        const double x = param_first ? p : other, y = param_first ? other : p;
        if (std::fabs(x - y) >= 0x1p977) continue;
        diff.check_diff(x, y, b);
    }

    const Tally* all[] = {&random, &engine, &tiny, &subq, &huge, &hard, &zero, &negzero, &diff};
    for (const Tally* t : all) t->print();
    return 0;
}
