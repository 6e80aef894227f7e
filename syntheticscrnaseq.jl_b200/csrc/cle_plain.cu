// Plain FP64 one-kernel-per-step CLE (the comparison baseline), the standalone
// capture kernels, the device Philox check and the pipe-throughput microkernels.
//
// The FP64 step kernel is a direct per-step formulation of cle.jl:78-121: one
// thread per (cell, gene), state in HBM, protein double-buffered because the
// regulation reads the previous step's proteins of other genes, and the
// reference's two-term A_pos*act + A_neg*rep contraction over the sparse edges.
// It consumes the same Philox increments as the fused kernel.
#include "cle_device.cuh"
#include "cle_internal.h"

namespace scrna {

__device__ __forceinline__ double pow_hill(double p, double n, int hill_int) {
    if (hill_int == 2) return p * p;
    return pow(p, n);
}

__global__ void __launch_bounds__(128) cle_plain_step_kernel(const PlainArgs a) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (c >= a.N) return;
    const Key key{a.key0, a.key1};
    const uint32_t gcell = (uint32_t)(a.cell_offset + c);
    const size_t idx = (size_t)g * a.N + c;
    const GeneRec gr = a.genes[g];
    const int s = a.step;

    // normals of this (cell, step, gene)
    const uint4 w = philox(gcell, (uint32_t)s, (uint32_t)(g >> 1), tagword(TAG_NORMAL, a.stream), key);
    const uint32_t w0 = (g & 1) ? w.z : w.x, w1 = (g & 1) ? w.w : w.y;
    // telegraph switching: the promoter switches when its waiting time runs out and draws
    // the next one from the spare bits of its normal words
    bool on = a.prom[idx];
    const int2 sw = a.NS[idx];
    if (s == sw.x) {
        on = !on;
        a.NS[idx] = switch_at(s, sw, switch_uniform(w0, w1), on, gr.inv_on, gr.inv_off);
        a.prom[idx] = on;
    }
    // reg = A_pos*act + A_neg*rep over the in-edges, from the previous step's proteins
    double s1 = 0.0, s2 = 0.0;
    for (int e = gr.in_begin; e < gr.in_end; ++e) {
        const int slot = __float_as_int(a.in_edge[e].y);
        const double pj = a.Pold[(size_t)a.reg_gene[slot] * a.N + c];
        const double pn = pow_hill(pj, a.hill_n, a.hill_n == 2.0 ? 2 : 0);
        const double den = __dadd_rn(pn, a.Kn);
        const double w = a.in_w64[e];
        if (w > 0.0) s1 = __dadd_rn(s1, __dmul_rn(w, __ddiv_rn(pn, den)));
        else s2 = __dadd_rn(s2, __dmul_rn(-w, __ddiv_rn(a.Kn, den)));
    }
    double reg = __dadd_rn(s1, s2);
    const int nab = gr.na_range >> 16, nac = gr.na_range & 0xFFFF;
    for (int e = nab; e < nab + nac; ++e) {
        const NonAdd na = a.na[e];
        double prod = 1.0;
        for (int t = na.src_begin; t < na.src_end; ++t) {
            const double pj = a.Pold[(size_t)a.reg_gene[a.na_src[t]] * a.N + c];
            const double pn = pow_hill(pj, a.hill_n, a.hill_n == 2.0 ? 2 : 0);
            const double act = __ddiv_rn(pn, __dadd_rn(pn, a.Kn));
            prod = na.kind == 0 ? __dmul_rn(prod, act) : __dmul_rn(prod, __dadd_rn(1.0, -act));
        }
        const double val = na.kind == 0 ? prod : __dadd_rn(1.0, -prod);
        reg = __dadd_rn(reg, __dmul_rn(a.na_coef64[e], val));
    }
    double zm, zp;
    box_muller_f64(w0, w1, &zm, &zp);

    double tx = __dadd_rn(reg, a.beta64[g]);
    if (!on) tx = 0.0;
    double mg = a.M[idx];
    const double pg = a.Pold[idx];
    double var_m = __dadd_rn(tx, __dmul_rn(a.mu_m, mg > 0.0 ? mg : 0.0));
    if (!(var_m > 0.0)) var_m = 0.0;
    const double nm = __dmul_rn(__dmul_rn(zm, a.sqrt_dt), sqrt(var_m));
    mg = __dadd_rn(__dadd_rn(mg, __dmul_rn(__dadd_rn(tx, -__dmul_rn(a.mu_m, mg)), a.dt)), nm);
    if (!(mg > 0.0)) mg = 0.0;
    double var_p = __dadd_rn(__dmul_rn(a.k_t, mg > 0.0 ? mg : 0.0), __dmul_rn(a.mu_p, pg > 0.0 ? pg : 0.0));
    if (!(var_p > 0.0)) var_p = 0.0;
    const double np_ = __dmul_rn(__dmul_rn(zp, a.sqrt_dt), sqrt(var_p));
    double pnew = __dadd_rn(__dadd_rn(pg, __dmul_rn(__dadd_rn(__dmul_rn(a.k_t, mg), -__dmul_rn(a.mu_p, pg)), a.dt)), np_);
    if (!(pnew > 0.0)) pnew = 0.0;
    a.M[idx] = mg;
    a.Pnew[idx] = pnew;
}

cudaError_t plain_step_launch(const PlainArgs& a, cudaStream_t st) {
    dim3 grid((unsigned)((a.N + 127) / 128), (unsigned)a.G);
    cle_plain_step_kernel<<<grid, 128, 0, st>>>(a);
    return cudaGetLastError();
}

// Initial FP64 state: ceil(steady state) and the initial promoter draws.
__global__ void plain_init_kernel(int G, int64_t N, int64_t cell_offset, const GeneInit* gi,
                                  const GeneRec* gr, uint32_t key0, uint32_t key1, uint32_t stream,
                                  double* M, double* P, uint8_t* prom, int2* NS) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (c >= N) return;
    const size_t idx = (size_t)g * N + c;
    M[idx] = (double)gi[g].m0;
    P[idx] = (double)gi[g].p0;
    bool on = true;
    if (gi[g].init_rand) {
        const uint4 w = philox((uint32_t)(cell_offset + c), 0u, (uint32_t)(g >> 2),
                               tagword(TAG_PROMOTER, stream), Key{key0, key1});
        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
        on = ws[g & 3] < gi[g].thr_init;
    }
    prom[idx] = on;
    int2 ns = make_int2(kNever, kNever);
    if (gr[g].inv_off == gr[g].inv_off) {
        const uint4 w = philox((uint32_t)(cell_offset + c), 0u, (uint32_t)g, tagword(TAG_SWITCH, stream),
                               Key{key0, key1});
        ns = fresh_switch(0, w.x, w.y, on, gr[g].inv_on, gr[g].inv_off);
    }
    NS[idx] = ns;
}

cudaError_t plain_init_launch(int G, int64_t N, int64_t cell_offset, const GeneInit* gi,
                              const GeneRec* gr, uint32_t key0, uint32_t key1, uint32_t stream,
                              double* M, double* P, uint8_t* prom, int2* NS, cudaStream_t st) {
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)G);
    plain_init_kernel<<<grid, 128, 0, st>>>(G, N, cell_offset, gi, gr, key0, key1, stream, M, P, prom, NS);
    return cudaGetLastError();
}

// Readout of an FP64 state ([G][N]) into the cells x G (x2) column-major output.
__global__ void plain_readout_kernel(int G, int64_t N, const double* M, const double* P,
                                     int readout, double* out) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (c >= N) return;
    const size_t idx = (size_t)g * N + c;
    if (readout == 0) out[idx] = M[idx];
    else if (readout == 1) out[idx] = P[idx];
    else { out[idx] = M[idx]; out[(size_t)(G + g) * N + c] = P[idx]; }
}

cudaError_t plain_readout_launch(int G, int64_t N, const double* M, const double* P, int readout,
                                 double* out, cudaStream_t st) {
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)G);
    plain_readout_kernel<<<grid, 128, 0, st>>>(G, N, M, P, readout, out);
    return cudaGetLastError();
}

// ---- capture (capture.jl:25-47) -------------------------------------------------------
__global__ void capture_eff_kernel(int64_t N, int64_t cell_offset, double mu_log, double sigma,
                                   uint32_t key0, uint32_t key1, uint32_t stream, double* eff) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= N) return;
    const uint4 w = philox((uint32_t)(cell_offset + c), 0u, 0u, tagword(TAG_EFFICIENCY, stream),
                           Key{key0, key1});
    double pe = exp(mu_log + sigma * box_muller_z0_f64(w.x, w.y));
    eff[c] = fmin(fmax(pe, 0.0), 1.0);
}

__global__ void capture_counts_kernel(int G, int64_t N, int64_t cell_offset, const double* X,
                                      const double* eff, uint32_t key0, uint32_t key1,
                                      uint32_t stream, int32_t* Y) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int g = blockIdx.y;
    if (c >= N) return;
    const size_t idx = (size_t)g * N + c;
    const double x = rint(X[idx]);
    const int64_t n = x > 0.0 ? (int64_t)x : 0;
    const double pe = eff[c];
    int64_t y = 0;
    if (n > 0 && pe != 0.0)
        y = binomial_capture(n, pe, Key{key0, key1}, stream, (uint32_t)(cell_offset + c), (uint32_t)g);
    Y[idx] = (int32_t)y;
}

cudaError_t capture_launch(int G, int64_t N, int64_t cell_offset, const double* X, double mu_log,
                           double sigma, uint32_t key0, uint32_t key1, uint32_t stream, double* eff,
                           int32_t* Y, cudaStream_t st) {
    capture_eff_kernel<<<(unsigned)((N + 127) / 128), 128, 0, st>>>(N, cell_offset, mu_log, sigma,
                                                                     key0, key1, stream, eff);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned)((N + 127) / 128), (unsigned)G);
    capture_counts_kernel<<<grid, 128, 0, st>>>(G, N, cell_offset, X, eff, key0, key1, stream, Y);
    return cudaGetLastError();
}

// ---- table of switch-uniform log2 values (switch_table.cuh) ------------------------------------
__global__ void switch_log2_init_kernel(float* tab, uint32_t n) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < n) tab[b] = own_log2f(switch_uniform_bits(b));
}

cudaError_t switch_log2_init_launch(float* tab, uint32_t n, cudaStream_t st) {
    switch_log2_init_kernel<<<(n + 255) / 256, 256, 0, st>>>(tab, n);
    return cudaGetLastError();
}

// ---- device Philox check ------------------------------------------------------------------
__global__ void philox_check_kernel(int n, const uint32_t* ctr, uint32_t k0, uint32_t k1,
                                    uint32_t* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 w = philox(ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3], Key{k0, k1});
    out[4 * i] = w.x; out[4 * i + 1] = w.y; out[4 * i + 2] = w.z; out[4 * i + 3] = w.w;
}

cudaError_t philox_check_launch(int n, const uint32_t* d_ctr, uint32_t k0, uint32_t k1,
                                uint32_t* d_out, cudaStream_t st) {
    philox_check_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, d_ctr, k0, k1, d_out);
    return cudaGetLastError();
}

// ---- pipe-throughput microkernels -----------------------------------------------------------
// Eight independent dependency chains per thread; the chain results are folded into a
// store guarded by an impossible condition so the work cannot be removed.
__global__ void __launch_bounds__(256) peak_fma_kernel(int iters, float seed, float* sink) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = seed + 0.001f * (threadIdx.x + k);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], 0.9999f, 0.0001f);
    }
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += x[k];
    if (acc == -1.2345f) sink[threadIdx.x] = acc;
}

__global__ void __launch_bounds__(256) peak_sfu_kernel(int iters, float seed, float* sink) {
    float x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = seed + 0.001f * (threadIdx.x + k);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float y;
                asm volatile("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x[k]));
                x[k] = y;
            }
    }
    float acc = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc += x[k];
    if (acc == -1.2345f) sink[threadIdx.x] = acc;
}

__global__ void __launch_bounds__(256) peak_int_kernel(int iters, uint32_t seed, float* sink) {
    uint32_t x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = seed + threadIdx.x * 7u + k;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int r = 0; r < 16; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = x[k] * x[k] + 0x7F4A7C15u;  // not foldable
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) acc ^= x[k];
    if (acc == 0x12345u) sink[threadIdx.x] = (float)acc;
}

// Philox4x32-10 throughput: four independent generator chains per thread (each block's
// output is the next counter), round keys from the kernel parameters as in the CLE kernels.
__global__ void __launch_bounds__(256) peak_philox_kernel(int iters, const KeySchedule ks, float* sink) {
    uint4 c[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = make_uint4(blockIdx.x, threadIdx.x, k, 0x01000000u);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k] = philox_rk(c[k].x, c[k].y, c[k].z, c[k].w, ks.rk0, ks.rk1);
    }
    uint32_t acc = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) acc ^= c[k].x ^ c[k].y ^ c[k].z ^ c[k].w;
    if (acc == 0x12345u) sink[threadIdx.x] = (float)acc;
}

// Philox4x32-10 calls executed per thread: 4 * iters.
cudaError_t peak_philox_launch(int blocks, int iters, float* sink, cudaStream_t st) {
    KeySchedule ks{};
    for (int r = 0; r < 10; ++r) {
        ks.rk0[r] = 0x243F6A88u + (uint32_t)r * 0x9E3779B9u;
        ks.rk1[r] = 0x85A308D3u + (uint32_t)r * 0xBB67AE85u;
    }
    peak_philox_kernel<<<blocks, 256, 0, st>>>(iters, ks, sink);
    return cudaGetLastError();
}

// ops executed per thread per iteration: 16 * 8
cudaError_t peak_launch(int which, int blocks, int iters, float* sink, cudaStream_t st) {
    if (which == 0) peak_fma_kernel<<<blocks, 256, 0, st>>>(iters, 1.0f, sink);
    else if (which == 1) peak_sfu_kernel<<<blocks, 256, 0, st>>>(iters, 1.5f, sink);
    else peak_int_kernel<<<blocks, 256, 0, st>>>(iters, 12345u, sink);
    return cudaGetLastError();
}

}  // namespace scrna
