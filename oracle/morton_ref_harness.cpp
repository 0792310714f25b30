// Test-only harness: drives mizuba's own 4-D Morton encoder
// (mizuba/detail/mortonND_LUT.h, MortonNDLutEncoder<4, 16, 8> as used by
// mizuba/detect_conjunctions_morton.cpp:102) compiled in place from the
// reference tree.  Reads quadruples of 16-bit field values from stdin and
// prints one decimal code per line.  Built by oracle/build.py into
// oracle/_ref/morton_ref only when the reference tree is mounted.
#include <cstdint>
#include <cstdio>

#include "mortonND_LUT.h"

int main()
{
    constexpr auto enc = mortonnd::MortonNDLutEncoder<4, 16, 8>();
    unsigned long long a, b, c, d;
    while (std::scanf("%llu %llu %llu %llu", &a, &b, &c, &d) == 4) {
        const std::uint64_t code = enc.Encode(a, b, c, d);
        std::printf("%llu\n", static_cast<unsigned long long>(code));
    }
    return 0;
}
