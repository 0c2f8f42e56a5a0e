// Harness around the reference's own CUDA PP kernel -- MEASUREMENT AND TEST
// INFRASTRUCTURE ONLY, never part of the product.
//
// The reference ships one GPU experiment, lcl_g_2.cu: updateKernel
// (lcl_g_2.cu:7-103) computes the short-range Yukawa-Ewald force on every
// particle from a linked-cell grid of floor(L/rc)^3 cells, each an array of
// 8-float slots (id, Z, x, y, z, ax, ay, az), one thread per particle and
// one 64-thread block per cell. Its main() reads a 1e7-particle file that
// the reference does not ship, so this harness builds the same cell arrays
// from given positions -- as lcl_g_2.cu:233-307 and :330-392 do -- and
// launches the kernel with the reference's own launch shape
// (lcl_g_2.cu:510-516: grid (512, ceil(Ncell/512)), 64 threads). The kernel
// is compiled from where the reference tree lies (the include below; the
// recipe in oracle/Makefile passes its path), with its main() renamed.
//
// The kernel's indexing hard-wires 37 slots per cell (thread t of cell c
// reads slot 37 c + t, lcl_g_2.cu:12-13,29-33), which is the capacity
// rc^3 + 10 of its main() only for rc = 3; the harness refuses any other
// capacity and any cell holding more particles than that, so every access
// the kernel makes stays inside the arrays it is given.
#include <cmath>
#include <cstdio>
#include <vector>

#define main lcl_g_2_reference_main
#include REF_LCL_G_2
#undef main

extern "C" int ref_update_kernel(int n, const float *pos, float L, float kappa, float G,
                                 float rc, int iters, float *acc_out, float *ms_per_launch)
{
    const float pi = 3.141592653589793f;
    const int nd = (int)floor(L / rc);
    if (nd < 3) return -1;  // fewer cells: the 27-cell stencil visits cells twice
    const int ncell = nd * nd * nd;
    const float rcw = L / nd;
    const int cap = (int)(pow(rc, 3) + 10.0);
    if (cap != 37) return -2;  // the kernel's slot indexing assumes 37 slots per cell
    const int atm = 8, blen = atm * cap;
    std::vector<float> bins((size_t)ncell * blen, -50.0f);  // the reference's empty mark
    std::vector<int> count(ncell, 0);
    for (int i = 0; i < n; ++i) {
        int cx = (int)floor(pos[3 * i] / rcw), cy = (int)floor(pos[3 * i + 1] / rcw),
            cz = (int)floor(pos[3 * i + 2] / rcw);
        if (cx < 0 || cy < 0 || cz < 0 || cx >= nd || cy >= nd || cz >= nd) return -3;
        const int c = cx + cy * nd + cz * nd * nd;
        if (count[c] >= cap) return -4;  // more particles than the kernel's slots
        float *slot = &bins[(size_t)c * blen + atm * count[c]];
        slot[0] = (float)i;
        slot[1] = 1.0f;
        slot[2] = pos[3 * i];
        slot[3] = pos[3 * i + 1];
        slot[4] = pos[3 * i + 2];
        slot[5] = slot[6] = slot[7] = 0.0f;
        ++count[c];
    }
    // 27 neighbour cells with periodic shifts, as lcl_g_2.cu:330-392
    const int clen = 27 * 4;
    std::vector<float> nl((size_t)ncell * clen);
    for (int c = 0; c < ncell; ++c) {
        const int cz = c / (nd * nd), cy = (c % (nd * nd)) / nd, cx = c % nd;
        int k = 0;
        for (int z = cz - 1; z < cz + 2; ++z)
            for (int y = cy - 1; y < cy + 2; ++y)
                for (int x = cx - 1; x < cx + 2; ++x) {
                    const int zs = z < 0 ? nd : (z >= nd ? -nd : 0);
                    const int ys = y < 0 ? nd : (y >= nd ? -nd : 0);
                    const int xs = x < 0 ? nd : (x >= nd ? -nd : 0);
                    nl[(size_t)c * clen + k] = (float)(x + xs + (y + ys) * nd + (z + zs) * nd * nd);
                    nl[(size_t)c * clen + k + 1] = x < 0 ? -L : (x >= nd ? L : 0.0f);
                    nl[(size_t)c * clen + k + 2] = y < 0 ? -L : (y >= nd ? L : 0.0f);
                    nl[(size_t)c * clen + k + 3] = z < 0 ? -L : (z >= nd ? L : 0.0f);
                    k += 4;
                }
    }
    int *d_count = nullptr;
    float *d_bins = nullptr, *d_nl = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rcode = 0;
    const dim3 grid(512, (unsigned)ceil(ncell / 512.0), 1), block(64, 1, 1);
    float ms = 0.0f;
    if (cudaMalloc(&d_count, ncell * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_bins, bins.size() * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_nl, nl.size() * sizeof(float)) != cudaSuccess) {
        rcode = -5;
        goto done;
    }
    cudaMemcpy(d_count, count.data(), ncell * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_bins, bins.data(), bins.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_nl, nl.data(), nl.size() * sizeof(float), cudaMemcpyHostToDevice);
    // one launch for the forces (the kernel adds into the slots)
    updateKernel<<<grid, block>>>(kappa, G, rc, pi, ncell, d_count, d_bins, blen, d_nl, clen);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        rcode = -6;
        goto done;
    }
    cudaMemcpy(bins.data(), d_bins, bins.size() * sizeof(float), cudaMemcpyDeviceToHost);
    for (int c = 0; c < ncell; ++c)
        for (int k = 0; k < count[c]; ++k) {
            const float *slot = &bins[(size_t)c * blen + atm * k];
            const int i = (int)slot[0];
            acc_out[3 * i] = slot[5];
            acc_out[3 * i + 1] = slot[6];
            acc_out[3 * i + 2] = slot[7];
        }
    // then `iters` timed launches, back to back
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int w = 0; w < 3; ++w)
        updateKernel<<<grid, block>>>(kappa, G, rc, pi, ncell, d_count, d_bins, blen, d_nl, clen);
    cudaEventRecord(e0);
    for (int it = 0; it < iters; ++it)
        updateKernel<<<grid, block>>>(kappa, G, rc, pi, ncell, d_count, d_bins, blen, d_nl, clen);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
        rcode = -6;
        goto done;
    }
    cudaEventElapsedTime(&ms, e0, e1);
    *ms_per_launch = ms / (iters > 0 ? iters : 1);
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(d_count);
    cudaFree(d_bins);
    cudaFree(d_nl);
    return rcode;
}
