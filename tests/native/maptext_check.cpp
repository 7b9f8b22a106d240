// Host check of the device map-text formatter (autogrid_b200/csrc/kernels/maptext.cuh)
// against the reference's own expression printed by glibc:
//   fabs(e) < PRECISION ? "0\n" : fprintf("%.3f\n", (float)round3dp(e))   (main.cpp:3481-3519)
//   round3dp(x) = round(x*1000.0L)/1000.0L                               (main.cpp:84-86)
// over seeded random values of every magnitude and the cases that decide the
// rounding: halves of round(), ties of "%.3f", doubles whose quotient falls
// halfway between two floats, |e| >= 2^53, overflow to inf, NaN, signed zero.
//
// usage: maptext_check <seed> <n_random>; exit 0 when every line matches.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <random>
#include <string>
#include <vector>

#include "kernels/maptext.cuh"

static std::string ref_line(int kind, double e)
{
    char buf[512];
    if (kind == agt::kCount) {
        std::snprintf(buf, sizeof buf, "%d\n", (int)e);
    } else if (kind == agt::kEnergy && std::fabs(e) < 0.0001) {
        std::snprintf(buf, sizeof buf, "0\n");
    } else {
        std::snprintf(buf, sizeof buf, "%.3f\n", (float)(std::round((long double)e * 1000.0L) / 1000.0L));
    }
    return buf;
}

static std::string got_line(int kind, double e)
{
    char buf[agt::kMaxLine + 1];
    const int n = agt::format_line(kind, e, buf);
    const int m = agt::format_line(kind, e, nullptr);
    if (n != m) return "<length mismatch>";
    return std::string(buf, buf + n);
}

int main(int argc, char **argv)
{
    const unsigned seed = argc > 1 ? (unsigned)std::atoi(argv[1]) : 1u;
    const long n_random = argc > 2 ? std::atol(argv[2]) : 1000000;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> u01(0.0, 1.0);
    std::vector<std::pair<int, double>> cases;
    auto add = [&](int kind, double e) { cases.emplace_back(kind, e); };
    auto both = [&](double e) {
        add(agt::kEnergy, e);
        add(agt::kFloating, e);
    };

    // fixed cases
    const double inf = std::numeric_limits<double>::infinity();
    const double fixed[] = {0.0, -0.0, 1e-4, -1e-4, 0.0005, -0.0005, 0.0625, -0.0625, 0.0015, 2.5e-4, -2.5e-4,
                            1e12, -1e12, 16384.0625, -16384.0625, 16384.0009765625, 9007199254740992.0,
                            9007199254740993.0 * 2, 1e15, 1e16, 1e20, 1e30, 3.4028234663852886e38,
                            3.4028235677973366e38, 3.5e38, 1e300, -1e300, inf, -inf,
                            std::numeric_limits<double>::quiet_NaN(), -std::numeric_limits<double>::quiet_NaN(),
                            4.9406564584124654e-324, -4.9406564584124654e-324, 2.2250738585072014e-308,
                            100000.0, 99999.9995, 0.9995, 1.0005, -1.0005, 123.4565, 8388608.5, 16777217.0};
    for (double e : fixed) {
        both(e);
        both(std::nextafter(e, inf));
        both(std::nextafter(e, -inf));
    }
    // counts
    for (int k = 0; k < 2000; k++) add(agt::kCount, (double)k);
    add(agt::kCount, 100000.0);
    add(agt::kCount, 2147483647.0);

    // halves of round(): e*1000 = k + 0.5 exactly (dyadic e), and their neighbours
    for (int i = 0; i < 200000; i++) {
        const int s = 1 + (int)(rng() % 14);
        const double j = (double)(int64_t)(rng() % (1ull << 30)) - (double)(1ull << 29);
        const double e = j / (double)(1ull << s);
        both(e);
        both(std::nextafter(e, inf));
        both(std::nextafter(e, -inf));
    }
    // decimal ticks k/1000 and (k+0.5)/1000 as parsed doubles, with neighbours
    for (int i = 0; i < 200000; i++) {
        const double k = (double)(int64_t)(rng() % 200000000ull) - 1e8;
        for (double e : {k / 1000.0, (k + 0.5) / 1000.0}) {
            both(e);
            both(std::nextafter(e, inf));
            both(std::nextafter(e, -inf));
        }
    }
    // quotients that fall halfway between two floats: m = odd 25-bit * 2^x,
    // m*1000 an integer for x >= -3
    for (int i = 0; i < 100000; i++) {
        const double odd = (double)((1ull << 24) | (rng() & ((1ull << 24) - 1)) | 1ull);
        const int x = -3 + (int)(rng() % 30);
        const double e = std::ldexp(odd, x - 1) * ((rng() & 1) ? -1.0 : 1.0);
        both(e);
        both(std::nextafter(e, inf));
    }
    // |e| in [2^43, 2^53): round(e*1000) above 2^53
    for (int i = 0; i < 100000; i++) {
        const double e = std::ldexp(1.0 + u01(rng), 43 + (int)(rng() % 10)) * ((rng() & 1) ? -1.0 : 1.0);
        both(e);
    }
    // log-uniform magnitudes, random signs, and map-like values
    for (long i = 0; i < n_random; i++) {
        const double mag = std::pow(10.0, -7.0 + 23.0 * u01(rng));
        both(((rng() & 1) ? -1.0 : 1.0) * mag);
        both(200.0 * (u01(rng) - 0.5));
        add(agt::kFloating, 20.0 * u01(rng));
    }

    long bad = 0;
    for (const auto &c : cases) {
        const std::string r = ref_line(c.first, c.second), g = got_line(c.first, c.second);
        if (r != g) {
            if (bad < 20) {
                std::string rr = r, gg = g;
                if (!rr.empty()) rr.pop_back();
                if (!gg.empty() && gg.back() == '\n') gg.pop_back();
                std::printf("kind %d e %.17g: reference \"%s\" got \"%s\"\n", c.first, c.second, rr.c_str(), gg.c_str());
            }
            bad++;
        }
    }
    std::printf("%zu cases, %ld mismatches\n", cases.size(), bad);
    return bad ? 1 : 0;
}
