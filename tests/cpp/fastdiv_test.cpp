// Host path of cn::FastDiv (cubismnova_b200/csrc/cn_fastdiv.h) against exact
// integer division: every divisor 1..4096 with all numerators below 2^16
// and at the edges of the range, plus seeded random divisors and numerators
// up to 2^31 - 1.  Exit status 0 = pass.
#include "cn_fastdiv.h"

#include <cstdint>
#include <cstdio>

static int failures = 0;

static void check(uint32_t d, int n)
{
    const cn::FastDiv f(d);
    const int want = (int)((uint32_t)n / d);
    if (f.div(n) != want && failures++ < 10)
        std::printf("FAILED d=%u n=%d: %d != %d\n", d, n, f.div(n), want);
}

int main()
{
    const int edges[] = {0, 1, 2, 3, 65535, 65536, 1 << 20, (1 << 30) - 1, 1 << 30, 2147483646, 2147483647};
    for (uint32_t d = 1; d <= 4096; ++d) {
        for (int n = 0; n < (1 << 16); n += (d < 64 ? 1 : 7)) check(d, n);
        for (int n : edges) check(d, n);
        for (int k = 1; k < 64; ++k) {
            const int64_t m = (int64_t)k * d;
            if (m - 1 < 2147483647) check(d, (int)(m - 1));
            if (m < 2147483647) check(d, (int)m);
        }
    }
    uint64_t s = 0x9E3779B97F4A7C15ull;
    auto next = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    };
    for (int i = 0; i < 2000000; ++i) {
        const uint32_t d = 1 + (uint32_t)(next() % 2147483647u);
        check(d, (int)(next() % 2147483648u));
    }
    std::printf("%s (%d failures)\n", failures ? "FAIL" : "PASS", failures);
    return failures ? 1 : 0;
}
