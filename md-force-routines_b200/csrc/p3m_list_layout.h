// Neighbour-list layout of the pair kernels, shared by the list builder (the
// writer), the pair loops and the inner-list store (the readers). Plain
// integer arithmetic, compiled for the device by nvcc and for the host by any
// C++17 compiler, so the host can check that every reader address is the
// writer's address of the same entry and that all of them stay inside the
// list array.
#pragma once

#ifdef __CUDACC__
#define P3M_LAYOUT_FN __host__ __device__ __forceinline__
#else
#define P3M_LAYOUT_FN inline
#endif

namespace p3m {

// Neighbour lists are padded with the particle's own index to a multiple of
// this many entries (a padded entry has r = 0 and adds nothing), so the FP32
// pair loop reads whole blocks of entries without a bounds test.
constexpr int PP_LIST_PAD = 16;

// List layout. A particle's entries come in blocks of PP_LIST_PAD = 16, and
// block b of the 32 consecutive sorted particles s >> 5 is stored as one
// group block of 512 entries (2 KB) at ((s >> 5) maxnb + 16 b) 32. Inside a
// group block the order follows the FP32 pair kernel with TPI = 2^lt lanes
// per particle: a pass takes STEP = UNR TPI entries of a particle (UNR =
// min(16 / TPI, 8)), lane `sub` entries v TPI + sub (v < UNR) as UNR / C
// chunks of C = min(UNR, 4) contiguous entries, and chunk i of all 32
// particles' lanes lies together -- so one vector load of a warp whose
// particles lie in one group reads 512 contiguous bytes (256 at TPI 8; a warp
// across two groups reads two runs), and the 16 entries of a particle's block
// lie within its group block (coalesced list writes). Lists are rebuilt
// whenever TPI changes. maxnb (entries per particle) is a multiple of 16.
P3M_LAYOUT_FN constexpr int pp_unr(int tpi) { return 16 / tpi < 8 ? 16 / tpi : 8; }
P3M_LAYOUT_FN constexpr int pp_chunk(int tpi) { return pp_unr(tpi) < 4 ? pp_unr(tpi) : 4; }
P3M_LAYOUT_FN constexpr int pp_step(int tpi) { return pp_unr(tpi) * tpi; }
// entries between a lane's consecutive chunks
P3M_LAYOUT_FN constexpr int list_cstride(int tpi) { return 32 * tpi * pp_chunk(tpi); }

// Writer side: list_index(s, e) = list_row(s) + list_col(e), the particle's
// part and the entry's part of the index of entry e of sorted particle s.
P3M_LAYOUT_FN int list_lc(int lt) { return (lt == 0 ? 3 : 4 - lt) < 2 ? 1 : 2; }  // log2 C
P3M_LAYOUT_FN long long list_row(int s, int maxnb, int lt)
{
    return (long long)(s >> 5) * maxnb * 32 + ((s & 31) << (lt + list_lc(lt)));
}
P3M_LAYOUT_FN int list_col(int e, int lt)
{
    const int lu = lt == 0 ? 3 : 4 - lt;  // log2 UNR
    const int ls = lu + lt;               // log2 STEP (3 or 4)
    const int lc = list_lc(lt);           // log2 C
    const int e16 = e & 15, pass = e16 >> ls, w = e16 & ((1 << ls) - 1);
    const int sub = w & ((1 << lt) - 1), v = w >> lt;
    const int chunk = (pass << (lu - lc)) + (v >> lc);
    return ((e & ~15) << 5) + (chunk << (5 + lt + lc)) + (sub << lc) + (v & ((1 << lc) - 1));
}
P3M_LAYOUT_FN long long list_index(int s, int e, int maxnb, int lt)
{
    return list_row(s, maxnb, lt) + list_col(e, lt);
}

// Reader side, for a lane `sub` of the TPI lanes of the particle in slot p32
// (s & 31) of group g (s >> 5). list_lane_at(list, ...): the lane's first
// chunk. Inside a particle's block b (entries 16 b .. 16 b + 15), chunk i of
// pass p holds entries 16 b + p STEP + (i C + c) TPI + sub, c < C, at
// list_block(b) + list_chunk(p, i) from there; list_pass_at(lane, k0) is the
// lane's chunk 0 of the pass that starts at entry k0 (a multiple of STEP).
// The _at forms advance a pointer (or any type with + long long) in the
// order the pair loops add the terms.
template <int TPI, typename P>
P3M_LAYOUT_FN P list_lane_at(P list, int g, int p32, int sub, int maxnb)
{
    return list + (long long)g * maxnb * 32 + (p32 * TPI + sub) * pp_chunk(TPI);
}
P3M_LAYOUT_FN long long list_block(int b) { return (long long)b * PP_LIST_PAD * 32; }
template <int TPI>
P3M_LAYOUT_FN int list_chunk(int p, int i)
{
    return (p * (pp_unr(TPI) / pp_chunk(TPI)) + i) * list_cstride(TPI);
}
template <int TPI, typename P>
P3M_LAYOUT_FN P list_pass_at(P lane, int k0)
{
    constexpr int STEP = pp_step(TPI), NCH = pp_unr(TPI) / pp_chunk(TPI);
    return lane + (long long)(k0 & ~15) * 32 + ((k0 & 15) / STEP) * NCH * list_cstride(TPI);
}

}  // namespace p3m
