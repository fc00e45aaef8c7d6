// Host-side check of the pressure solve's chunk rule (ariel_b200/csrc/pcg.cuh): for every scene
// size, no FLUID count can cut the scene into more chunks than chunk_bound() reserved partial-sum
// slots for (the solve writes one slot per chunk), and every chosen chunk size is a power of two
// within the documented range.  Runs on the CPU only; prints "ok" and exits 0 when all hold.
#include <cstdio>

#include "pcg.cuh"

using ariel::chunk_bound;
using ariel::chunk_shift;

static int check(long long cells, long long nf) {
    const int sh = chunk_shift(nf);
    if (sh < ariel::kChunkMinShift || sh > ariel::kChunkMaxShift) {
        std::printf("shift %d out of range for %lld FLUID cells\n", sh, nf);
        return 1;
    }
    const long long chunks = (nf + (1ll << sh) - 1) >> sh;
    if (chunks > chunk_bound(cells)) {
        std::printf("%lld FLUID cells of %lld: %lld chunks > bound %lld\n", nf, cells, chunks, chunk_bound(cells));
        return 1;
    }
    // a smaller chunk would have been chosen if it kept the count within the target
    if (sh > ariel::kChunkMinShift && ((nf + (1ll << (sh - 1)) - 1) >> (sh - 1)) <= ariel::kChunkTarget) {
        std::printf("%lld FLUID cells: shift %d is not the smallest within the target\n", nf, sh);
        return 1;
    }
    return 0;
}

int main() {
    int bad = 0;
    // every FLUID count of every cubic grid up to 96^3, all counts
    for (long long n = 1; n <= 96 && !bad; ++n)
        for (long long nf = 0; nf <= n * n * n && !bad; ++nf) bad |= check(n * n * n, nf);
    // larger grids up to 1024^3: counts around every power of two and chunk-size threshold, and
    // a stride through the whole range
    for (long long n = 97; n <= 1024 && !bad; n += 7) {
        const long long cells = n * n * n;
        for (long long p = 1; p <= cells && !bad; p <<= 1)
            for (long long d = -3; d <= 3 && !bad; ++d)
                if (p + d >= 0 && p + d <= cells) bad |= check(cells, p + d);
        for (int t = 1; t <= 4 && !bad; ++t) {
            const long long edge = ariel::kChunkTarget << (ariel::kChunkMinShift + t - 1);
            for (long long d = -3; d <= 3 && !bad; ++d)
                if (edge + d >= 0 && edge + d <= cells) bad |= check(cells, edge + d);
        }
        for (long long nf = 0; nf <= cells && !bad; nf += cells / 997 + 1) bad |= check(cells, nf);
        if (!bad) bad |= check(cells, cells);
    }
    if (!bad) std::printf("ok\n");
    return bad;
}
