// Host check of the neighbour-list layout the pair kernels use
// (md-force-routines_b200/csrc/p3m_list_layout.h, compiled here by the host
// compiler from the same header nvcc compiles into the kernels).
//
// For every threads-per-particle setting (TPI = 2^lt, lt = 0..3), several
// list capacities maxnb (multiples of 16) and a few 32-particle groups:
//  1. the writer's index list_index(s, e) is a bijection of {s} x [0, maxnb)
//     onto [0, 32 groups maxnb): no two entries share a slot, none is outside
//     the list array (sized n_groups * 32 * maxnb by the host);
//  2. the 16 entries of a particle's block b lie inside its group block of
//     512 entries at ((s >> 5) maxnb + 16 b) 32;
//  3. the pair loops' reads (list_lane_at, then list_pass_at per pass, then
//     chunk i at list_cstride i, C entries each) reach exactly the writer's
//     slot of entry k0 + (i C + c) TPI + sub, and the lanes of a particle
//     together read each of its entries once;
//  4. every chunk starts on a multiple of C entries (the int4 / int2 vector
//     loads and stores are aligned when the list array is);
//  5. the inner-list store (list_lane_at + list_block + list_chunk) writes
//     entry 16 blk + p STEP + (i C + c) TPI + sub at the writer's slot;
//  6. one chunk of a warp's 32 lanes is 32 C contiguous entries (a single
//     512-byte, or 256-byte at TPI 8, access) when the warp's particles lie
//     in one group; a replica that starts inside a group (particle offsets
//     are cumulative N) has warps across two groups, which read two runs.
// Prints "ok <checks>" and exits 0, or prints the first mismatch and exits 1.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "p3m_list_layout.h"

using namespace p3m;

namespace {

// PLANT_SKEW (a test of this check, default 0) moves every reader address
// by that many entries, which checks 3 to 5 must catch.
#ifndef PLANT_SKEW
#define PLANT_SKEW 0
#endif

struct Addr {  // an address as a plain offset, added in the kernels' order
    long long v;
};
Addr operator+(Addr a, long long d) { return Addr{a.v + d + PLANT_SKEW}; }

long long g_checks = 0;

#define CHECK(cond, ...)                                     \
    do {                                                     \
        ++g_checks;                                          \
        if (!(cond)) {                                       \
            std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
            std::printf(__VA_ARGS__);                        \
            std::printf("\n");                               \
            std::exit(1);                                    \
        }                                                    \
    } while (0)

template <int TPI>
void check(int maxnb, int groups)
{
    constexpr int lt = TPI == 1 ? 0 : TPI == 2 ? 1 : TPI == 4 ? 2 : 3;
    constexpr int UNR = pp_unr(TPI), STEP = pp_step(TPI), C = pp_chunk(TPI), NCH = UNR / C;
    constexpr int CSTRIDE = list_cstride(TPI);
    static_assert(UNR % C == 0 && PP_LIST_PAD % STEP == 0 && STEP <= PP_LIST_PAD, "layout");
    CHECK(maxnb % PP_LIST_PAD == 0, "maxnb %d not a multiple of 16", maxnb);
    CHECK((1 << list_lc(lt)) == C, "list_lc(%d) against C = %d", lt, C);

    const int ns = 32 * groups;
    const long long total = (long long)ns * maxnb;
    std::vector<int> owner(total, -1);  // slot -> s * maxnb + e

    // 1 and 2: the writer
    for (int s = 0; s < ns; ++s)
        for (int e = 0; e < maxnb; ++e) {
            const long long x = list_index(s, e, maxnb, lt);
            CHECK(x >= 0 && x < total, "TPI %d maxnb %d: s %d e %d -> %lld outside [0, %lld)", TPI,
                  maxnb, s, e, x, total);
            CHECK(owner[x] < 0, "TPI %d maxnb %d: s %d e %d -> %lld taken by entry %d", TPI, maxnb, s,
                  e, x, owner[x]);
            owner[x] = s * maxnb + e;
            const long long gb = ((long long)(s >> 5) * maxnb + 16 * (e >> 4)) * 32;
            CHECK(x >= gb && x < gb + 512, "TPI %d: s %d e %d -> %lld outside its group block %lld",
                  TPI, s, e, x, gb);
            CHECK(list_row(s, maxnb, lt) + list_col(e, lt) == x, "list_index != row + col");
        }

    // 3 and 4: the pair loops' reads
    std::vector<int> seen(maxnb);
    for (int s = 0; s < ns; ++s) {
        std::fill(seen.begin(), seen.end(), 0);
        for (int sub = 0; sub < TPI; ++sub) {
            const Addr lane = list_lane_at<TPI>(Addr{0}, s >> 5, s & 31, sub, maxnb);
            for (int k0 = 0; k0 < maxnb; k0 += STEP) {
                const Addr lp = list_pass_at<TPI>(lane, k0);
                for (int i = 0; i < NCH; ++i) {
                    const long long chunk = lp.v + (long long)i * CSTRIDE;
                    CHECK(chunk % C == 0, "TPI %d: chunk at %lld not aligned to %d", TPI, chunk, C);
                    for (int c = 0; c < C; ++c) {
                        const int e = k0 + (i * C + c) * TPI + sub;
                        CHECK(e < maxnb, "TPI %d: read entry %d beyond maxnb %d", TPI, e, maxnb);
                        CHECK(chunk + c == list_index(s, e, maxnb, lt),
                              "TPI %d maxnb %d: s %d sub %d k0 %d chunk %d c %d reads %lld, entry %d is "
                              "at %lld",
                              TPI, maxnb, s, sub, k0, i, c, chunk + c, e, list_index(s, e, maxnb, lt));
                        ++seen[e];
                    }
                }
            }
        }
        for (int e = 0; e < maxnb; ++e)
            CHECK(seen[e] == 1, "TPI %d: s %d entry %d read %d times", TPI, s, e, seen[e]);
    }

    // 5: the inner-list store (maxnb doubles as the inner capacity)
    for (int s = 0; s < ns; ++s)
        for (int sub = 0; sub < TPI; ++sub) {
            const Addr og = list_lane_at<TPI>(Addr{0}, s >> 5, s & 31, sub, maxnb);
            for (int blk = 0; blk < maxnb / PP_LIST_PAD; ++blk)
                for (int p = 0; p < PP_LIST_PAD / STEP; ++p)
                    for (int i = 0; i < NCH; ++i) {
                        const long long dst = (og + list_block(blk)).v + list_chunk<TPI>(p, i);
                        CHECK(dst % C == 0, "TPI %d: store at %lld not aligned", TPI, dst);
                        for (int c = 0; c < C; ++c) {
                            const int e = blk * PP_LIST_PAD + p * STEP + (i * C + c) * TPI + sub;
                            CHECK(dst + c == list_index(s, e, maxnb, lt),
                                  "TPI %d: store of s %d entry %d at %lld, writer's slot %lld", TPI, s, e,
                                  dst + c, list_index(s, e, maxnb, lt));
                        }
                    }
        }

    // 6: one chunk of a warp is contiguous
    constexpr int PPW = 32 / TPI;
    for (int g = 0; g < groups; ++g)
        for (int w = 0; w < TPI; ++w)  // warps of a 32-particle group
            for (int k0 = 0; k0 < maxnb; k0 += STEP)
                for (int i = 0; i < NCH; ++i) {
                    long long lo = -1, hi = -1;
                    for (int p = 0; p < PPW; ++p)
                        for (int sub = 0; sub < TPI; ++sub) {
                            const int s = 32 * g + PPW * w + p;
                            const long long a =
                                list_pass_at<TPI>(list_lane_at<TPI>(Addr{0}, s >> 5, s & 31, sub, maxnb),
                                                  k0).v +
                                (long long)i * CSTRIDE;
                            lo = lo < 0 || a < lo ? a : lo;
                            hi = a + C - 1 > hi ? a + C - 1 : hi;
                        }
                    CHECK(hi - lo + 1 == 32 * C, "TPI %d: warp %d pass %d chunk %d spans %lld entries",
                          TPI, w, k0, i, hi - lo + 1);
                }
}

}  // namespace

int main()
{
    const int caps[] = {16, 32, 48, 64, 272, 400, 2048};
    for (int maxnb : caps) {
        const int groups = maxnb > 1000 ? 2 : 3;
        check<1>(maxnb, groups);
        check<2>(maxnb, groups);
        check<4>(maxnb, groups);
        check<8>(maxnb, groups);
    }
    std::printf("ok %lld\n", g_checks);
    return 0;
}
