// Host-side check of the pressure solve's chunk rule (ariel_b200/csrc/pcg.cuh): for every scene
// size, no FLUID count can cut the scene into more chunks than chunk_bound() reserved partial-sum
// slots for (the solve writes one slot per chunk), and every chosen chunk size is a multiple of
// kChunkAlign within [kChunkMin, kChunkMax] that spreads the scene over at most kChunkTarget
// chunks unless the size is capped.  Runs on the CPU only; prints "ok" and exits 0 when all hold.
#include <cstdio>

#include "pcg.cuh"

using ariel::chunk_bound;
using ariel::chunk_size;

static int check(long long cells, long long nf) {
    const long long cs = chunk_size(nf);
    if (cs < ariel::kChunkMin || cs > ariel::kChunkMax || cs % ariel::kChunkAlign != 0) {
        std::printf("chunk size %lld out of range for %lld FLUID cells\n", cs, nf);
        return 1;
    }
    const long long chunks = (nf + cs - 1) / cs;
    if (chunks > chunk_bound(cells)) {
        std::printf("%lld FLUID cells of %lld: %lld chunks > bound %lld\n", nf, cells, chunks, chunk_bound(cells));
        return 1;
    }
    if (cs < ariel::kChunkMax && chunks > ariel::kChunkTarget) {
        std::printf("%lld FLUID cells: %lld chunks of %lld exceed the target\n", nf, chunks, cs);
        return 1;
    }
    // the size is the smallest aligned one within the target (or the floor)
    if (cs > ariel::kChunkMin && cs < ariel::kChunkMax &&
        (nf + cs - ariel::kChunkAlign - 1) / (cs - ariel::kChunkAlign) <= ariel::kChunkTarget) {
        std::printf("%lld FLUID cells: size %lld is not the smallest within the target\n", nf, cs);
        return 1;
    }
    return 0;
}

int main() {
    int bad = 0;
    // every FLUID count of every cubic grid up to 96^3, all counts
    for (long long n = 1; n <= 96 && !bad; ++n)
        for (long long nf = 0; nf <= n * n * n && !bad; ++nf) bad |= check(n * n * n, nf);
    // larger grids up to 1024^3: counts around every power of two and every size threshold, and a
    // stride through the whole range
    for (long long n = 97; n <= 1024 && !bad; n += 7) {
        const long long cells = n * n * n;
        for (long long p = 1; p <= cells && !bad; p <<= 1)
            for (long long d = -3; d <= 3 && !bad; ++d)
                if (p + d >= 0 && p + d <= cells) bad |= check(cells, p + d);
        for (long long cs = ariel::kChunkMin; cs <= ariel::kChunkMax && !bad; cs += ariel::kChunkAlign) {
            const long long edge = ariel::kChunkTarget * cs;
            for (long long d = -3; d <= 3 && !bad; ++d)
                if (edge + d >= 0 && edge + d <= cells) bad |= check(cells, edge + d);
        }
        for (long long nf = 0; nf <= cells && !bad; nf += cells / 997 + 1) bad |= check(cells, nf);
        if (!bad) bad |= check(cells, cells);
    }
    if (!bad) std::printf("ok\n");
    return bad;
}
