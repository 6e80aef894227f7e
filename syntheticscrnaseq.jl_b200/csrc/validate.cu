// On-device validation reductions over a state's results (src/validate.jl:14-77,
// src/analytical.jl:35-95 are the host-side formulas they feed), and the 10x Matrix Market
// writer of captured count matrices (the format experiments/compare_real_scrnaseq.jl:69-93
// reads).  The results stay on the device; only per-column summaries, or the nonzero
// entries of a slice of cells, cross to the host.
//
//   scrna_state_moments    per-column mean and unbiased variance, two passes in FP64
//   scrna_state_ks         per-column two-sample Kolmogorov-Smirnov statistic of two states
//                          (the merge walk of validate.jl:14-41, evaluated at every sample
//                          by binary search in the other sorted sample)
//   scrna_state_histogram  counts of the rounded values of one column
//   scrna_state_write_mtx  matrix.mtx (genes x cells, 1-based coordinates, integer), genes.tsv,
//                          barcodes.tsv; nonzeros compacted on the device slice by slice
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include <cub/device/device_segmented_sort.cuh>

#include "capi_internal.h"
#include "nvtx_range.h"

namespace scrna {
namespace {

// Column `col` of a cells x cols column-major matrix is contiguous: element (c, col) at col*N+c.
template <class T>
__global__ void column_moments_kernel(const T* X, int64_t N, double* mean, double* m2) {
    const int col = blockIdx.x;
    const T* x = X + (size_t)col * N;
    __shared__ double red[32];
    auto block_sum = [&](double v) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        double t = 0.0;
        if (threadIdx.x < 32) {
            t = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
        }
        __syncthreads();
        return t;  // valid in thread 0
    };
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) s += (double)x[i];
    s = block_sum(s);
    __shared__ double mu;
    if (threadIdx.x == 0) mu = s / (double)N;
    __syncthreads();
    const double m = mu;
    double q = 0.0;
    for (int64_t i = threadIdx.x; i < N; i += blockDim.x) {
        const double d = (double)x[i] - m;
        q += d * d;
    }
    q = block_sum(q);
    if (threadIdx.x == 0) {
        mean[col] = m;
        m2[col] = q;
    }
}

template <class T>
__global__ void to_double_kernel(const T* in, int64_t n, double* out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (double)in[i];
}

// Number of elements of sorted s[0, n) that are < v (strict) or <= v.
__device__ __forceinline__ int64_t count_below(const double* s, int64_t n, double v, bool inclusive) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (inclusive ? (s[mid] <= v) : (s[mid] < v)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// The walk of validate.jl:14-41 takes x before y on ties: right after it takes the i-th x
// (0-based) it has taken the y's below x_i, right after the j-th y the x's up to y_j.
// Every step's |ecdf_x - ecdf_y| is evaluated here; the column maximum is kept with an
// atomic max on the bits of the nonnegative double.
__global__ void ks_kernel(const double* sx, int64_t nx, const double* sy, int64_t ny, unsigned long long* dmax) {
    const int col = blockIdx.y;
    const double* x = sx + (size_t)col * nx;
    const double* y = sy + (size_t)col * ny;
    double d = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nx + ny; k += (int64_t)gridDim.x * blockDim.x) {
        double ex, ey;
        if (k < nx) {
            ex = (double)(k + 1) / (double)nx;
            ey = (double)count_below(y, ny, x[k], false) / (double)ny;
        } else {
            const int64_t j = k - nx;
            ex = (double)count_below(x, nx, y[j], true) / (double)nx;
            ey = (double)(j + 1) / (double)ny;
        }
        d = fmax(d, fabs(ex - ey));
    }
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xFFFFFFFFu, d, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&dmax[col], (unsigned long long)__double_as_longlong(d));
}

template <class T>
__global__ void histogram_kernel(const T* x, int64_t N, int nbins, unsigned long long* hist) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double v = rint((double)x[i]);
        v = fmin(fmax(v, 0.0), (double)(nbins - 1));
        atomicAdd(&hist[(int)v], 1ull);
    }
}

// Nonzeros per cell of cells [c0, c0 + nc) of a cells x G column-major int32 matrix.
__global__ void mtx_count_kernel(const int32_t* Y, int64_t N, int G, int64_t c0, int64_t nc, int32_t* cnt) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    int32_t n = 0;
    for (int g = 0; g < G; ++g) n += Y[(size_t)g * N + c0 + k] != 0;
    cnt[k] = n;
}

// Entries (gene, cell, count) of the slice, cell-major with genes ascending, at the offsets
// of the exclusive scan `off` of the counts.
__global__ void mtx_fill_kernel(const int32_t* Y, int64_t N, int G, int64_t c0, int64_t nc, const int64_t* off,
                                int32_t* gene, int32_t* count) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nc) return;
    int64_t o = off[k];
    for (int g = 0; g < G; ++g) {
        const int32_t v = Y[(size_t)g * N + c0 + k];
        if (v != 0) { gene[o] = g; count[o] = v; ++o; }
    }
}

int cols_of(const scrna_state* st) { return st->G * (st->readout == SCRNA_READOUT_BOTH ? 2 : 1); }

// Device data and column count of a state's readout (source 0, FP64) or counts (source 1, int32).
int source_of(const scrna_state* st, int source, const void** data, int* cols) {
    if (source == 0) {
        if (!st->out.p) return fail(SCRNA_EINVAL, "the state has not been run");
        *data = st->out.p;
        *cols = cols_of(st);
    } else if (source == 1) {
        if (!st->have_counts || !st->counts.p) return fail(SCRNA_EINVAL, "the state's last run had no capture");
        *data = st->counts.p;
        *cols = st->G;
    } else {
        return fail(SCRNA_EINVAL, "source must be 0 (readout) or 1 (counts)");
    }
    return SCRNA_OK;
}

// Sorted copy (FP64) of every column of a state's source.
int sorted_columns(scrna_ctx* ctx, const scrna_state* st, int source, DevBuf& out, int* cols) {
    const void* data;
    if (int r = source_of(st, source, &data, cols)) return r;
    const int64_t N = st->N, total = N * *cols;
    DevBuf tmp;
    CU(tmp.ensure((size_t)total * 8));
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (source == 0) CU(cudaMemcpyAsync(tmp.p, data, (size_t)total * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    else to_double_kernel<int32_t><<<blocks, 256, 0, ctx->stream>>>(static_cast<const int32_t*>(data), total, tmp.as<double>());
    CU(cudaGetLastError());
    std::vector<int64_t> offs(*cols + 1);
    for (int c = 0; c <= *cols; ++c) offs[c] = (int64_t)c * N;
    DevBuf d_offs;
    CU(d_offs.ensure(offs.size() * 8));
    CU(cudaMemcpyAsync(d_offs.p, offs.data(), offs.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    CU(out.ensure((size_t)total * 8));
    size_t tmp_bytes = 0;
    CU(cub::DeviceSegmentedSort::SortKeys(nullptr, tmp_bytes, tmp.as<double>(), out.as<double>(), total, *cols,
                                          d_offs.as<int64_t>(), d_offs.as<int64_t>() + 1, ctx->stream));
    DevBuf work;
    CU(work.ensure(std::max<size_t>(tmp_bytes, 16)));
    CU(cub::DeviceSegmentedSort::SortKeys(work.p, tmp_bytes, tmp.as<double>(), out.as<double>(), total, *cols,
                                          d_offs.as<int64_t>(), d_offs.as<int64_t>() + 1, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));  // the temporaries go out of scope here
    ctx->launches += 3;
    return SCRNA_OK;
}

}  // namespace
}  // namespace scrna

using namespace scrna;

extern "C" int scrna_state_moments(scrna_ctx* ctx, scrna_state* st, int32_t source, double* mean, double* var) {
    NvtxRange nvtx_range_("scrna_state_moments");
    if (!ctx || !st) return fail(SCRNA_EINVAL, "NULL argument");
    if (int r = set_device(ctx)) return r;
    const void* data;
    int cols;
    if (int r = source_of(st, source, &data, &cols)) return r;
    DevBuf d;
    CU(d.ensure((size_t)cols * 16));
    double* dm = d.as<double>();
    if (source == 0) column_moments_kernel<double><<<cols, 256, 0, ctx->stream>>>(static_cast<const double*>(data), st->N, dm, dm + cols);
    else column_moments_kernel<int32_t><<<cols, 256, 0, ctx->stream>>>(static_cast<const int32_t*>(data), st->N, dm, dm + cols);
    CU(cudaGetLastError());
    ctx->launches++;
    std::vector<double> h((size_t)cols * 2);
    CU(cudaMemcpyAsync(h.data(), dm, (size_t)cols * 16, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += (int64_t)cols * 16;
    for (int c = 0; c < cols; ++c) {
        if (mean) mean[c] = h[c];
        if (var) var[c] = st->N > 1 ? h[cols + c] / (double)(st->N - 1) : 0.0;
    }
    return SCRNA_OK;
}

extern "C" int scrna_state_ks(scrna_ctx* ctx, scrna_state* a, scrna_state* b, int32_t source, double* D) {
    NvtxRange nvtx_range_("scrna_state_ks");
    if (!ctx || !a || !b || !D) return fail(SCRNA_EINVAL, "NULL argument");
    if (int r = set_device(ctx)) return r;
    DevBuf sa, sb;
    int ca, cb;
    if (int r = sorted_columns(ctx, a, source, sa, &ca)) return r;
    if (int r = sorted_columns(ctx, b, source, sb, &cb)) return r;
    if (ca != cb) return fail(SCRNA_EINVAL, "the states have %d and %d columns", ca, cb);
    DevBuf dmax;
    CU(dmax.ensure((size_t)ca * 8));
    CU(cudaMemsetAsync(dmax.p, 0, (size_t)ca * 8, ctx->stream));
    const int64_t per_col = a->N + b->N;
    dim3 grid((unsigned)std::min<int64_t>((per_col + 255) / 256, 64), (unsigned)ca);
    ks_kernel<<<grid, 256, 0, ctx->stream>>>(sa.as<double>(), a->N, sb.as<double>(), b->N,
                                             dmax.as<unsigned long long>());
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaMemcpyAsync(D, dmax.p, (size_t)ca * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += (int64_t)ca * 8;
    return SCRNA_OK;
}

extern "C" int scrna_state_histogram(scrna_ctx* ctx, scrna_state* st, int32_t source, int32_t column, int32_t nbins,
                                     int64_t* hist) {
    NvtxRange nvtx_range_("scrna_state_histogram");
    if (!ctx || !st || !hist) return fail(SCRNA_EINVAL, "NULL argument");
    if (nbins <= 0) return fail(SCRNA_EINVAL, "nbins must be positive");
    if (int r = set_device(ctx)) return r;
    const void* data;
    int cols;
    if (int r = source_of(st, source, &data, &cols)) return r;
    if (column < 0 || column >= cols) return fail(SCRNA_EINVAL, "column %d out of range (%d columns)", column, cols);
    DevBuf h;
    CU(h.ensure((size_t)nbins * 8));
    CU(cudaMemsetAsync(h.p, 0, (size_t)nbins * 8, ctx->stream));
    const unsigned blocks = (unsigned)std::min<int64_t>((st->N + 255) / 256, 1024);
    if (source == 0)
        histogram_kernel<double><<<blocks, 256, 0, ctx->stream>>>(static_cast<const double*>(data) + (size_t)column * st->N,
                                                                  st->N, nbins, h.as<unsigned long long>());
    else
        histogram_kernel<int32_t><<<blocks, 256, 0, ctx->stream>>>(static_cast<const int32_t*>(data) + (size_t)column * st->N,
                                                                   st->N, nbins, h.as<unsigned long long>());
    CU(cudaGetLastError());
    ctx->launches++;
    CU(cudaMemcpyAsync(hist, h.p, (size_t)nbins * 8, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    ctx->d2h_bytes += (int64_t)nbins * 8;
    return SCRNA_OK;
}

extern "C" int scrna_state_write_mtx(scrna_ctx* ctx, scrna_state* st, const char* dir, const char* const* gene_names,
                                     const char* barcode_prefix) {
    NvtxRange nvtx_range_("scrna_state_write_mtx");
    if (!ctx || !st || !dir) return fail(SCRNA_EINVAL, "NULL argument");
    if (int r = set_device(ctx)) return r;
    const void* data;
    int cols;
    if (int r = source_of(st, 1, &data, &cols)) return r;
    const int32_t* Y = static_cast<const int32_t*>(data);
    const int G = st->G;
    const int64_t N = st->N;
    const std::string d(dir);
    // pass 1: nonzeros per cell, for the header
    const int64_t slice = std::min<int64_t>(N, 1 << 16);
    DevBuf cnt, off, gene, count;
    CU(cnt.ensure((size_t)slice * 4));
    std::vector<int32_t> hc((size_t)slice);
    std::vector<int64_t> nnz_of_slice;
    int64_t nnz = 0;
    for (int64_t c0 = 0; c0 < N; c0 += slice) {
        const int64_t nc = std::min(slice, N - c0);
        mtx_count_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, ctx->stream>>>(Y, N, G, c0, nc, cnt.as<int32_t>());
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(hc.data(), cnt.p, (size_t)nc * 4, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        int64_t s = 0;
        for (int64_t k = 0; k < nc; ++k) s += hc[k];
        nnz_of_slice.push_back(s);
        nnz += s;
        ctx->launches++;
    }
    FILE* f = std::fopen((d + "/matrix.mtx").c_str(), "wb");
    if (!f) return fail(SCRNA_EINVAL, "cannot write %s/matrix.mtx", dir);
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate integer general\n%%metadata_json: {\"software\": \"libscrna_cle\"}\n");
    std::fprintf(f, "%d %lld %lld\n", G, (long long)N, (long long)nnz);
    // pass 2: per slice, offsets by an exclusive scan of the counts on the host, the entries
    // compacted on the device, then formatted in cell order
    CU(off.ensure((size_t)slice * 8));
    std::vector<int64_t> ho((size_t)slice);
    std::vector<int32_t> hg, hv;
    std::string text;
    int si = 0;
    int rc = SCRNA_OK;
    for (int64_t c0 = 0; c0 < N && rc == SCRNA_OK; c0 += slice, ++si) {
        const int64_t nc = std::min(slice, N - c0);
        const int64_t m = nnz_of_slice[si];
        if (m == 0) continue;
        mtx_count_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, ctx->stream>>>(Y, N, G, c0, nc, cnt.as<int32_t>());
        cudaError_t e = cudaMemcpyAsync(hc.data(), cnt.p, (size_t)nc * 4, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { rc = fail(SCRNA_ECUDA, "mtx count: %s", cudaGetErrorString(e)); break; }
        int64_t run = 0;
        for (int64_t k = 0; k < nc; ++k) { ho[k] = run; run += hc[k]; }
        if ((e = gene.ensure((size_t)m * 4)) != cudaSuccess || (e = count.ensure((size_t)m * 4)) != cudaSuccess ||
            (e = cudaMemcpyAsync(off.p, ho.data(), (size_t)nc * 8, cudaMemcpyHostToDevice, ctx->stream)) != cudaSuccess) {
            rc = fail(SCRNA_ECUDA, "mtx buffers: %s", cudaGetErrorString(e));
            break;
        }
        mtx_fill_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, ctx->stream>>>(Y, N, G, c0, nc, off.as<int64_t>(),
                                                                              gene.as<int32_t>(), count.as<int32_t>());
        hg.resize((size_t)m);
        hv.resize((size_t)m);
        if ((e = cudaMemcpyAsync(hg.data(), gene.p, (size_t)m * 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hv.data(), count.p, (size_t)m * 4, cudaMemcpyDeviceToHost, ctx->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(ctx->stream)) != cudaSuccess) {
            rc = fail(SCRNA_ECUDA, "mtx entries: %s", cudaGetErrorString(e));
            break;
        }
        ctx->launches += 2;
        ctx->d2h_bytes += (int64_t)nc * 4 + m * 8;
        text.clear();
        char line[48];
        int64_t k = 0;
        for (int64_t c = 0; c < nc; ++c)
            for (int32_t j = 0; j < hc[c]; ++j, ++k) {
                const int len = std::snprintf(line, sizeof line, "%d %lld %d\n", hg[k] + 1, (long long)(c0 + c + 1), hv[k]);
                text.append(line, (size_t)len);
            }
        if (std::fwrite(text.data(), 1, text.size(), f) != text.size()) rc = fail(SCRNA_EINVAL, "short write to %s", dir);
    }
    if (std::fclose(f) != 0 && rc == SCRNA_OK) rc = fail(SCRNA_EINVAL, "cannot close %s/matrix.mtx", dir);
    if (rc != SCRNA_OK) return rc;
    // features (id and name, tab-separated, as 10x writes them) and barcodes
    FILE* fg = std::fopen((d + "/genes.tsv").c_str(), "wb");
    FILE* fb = std::fopen((d + "/barcodes.tsv").c_str(), "wb");
    if (!fg || !fb) {
        if (fg) std::fclose(fg);
        if (fb) std::fclose(fb);
        return fail(SCRNA_EINVAL, "cannot write genes.tsv / barcodes.tsv in %s", dir);
    }
    for (int g = 0; g < G; ++g) {
        if (gene_names && gene_names[g]) std::fprintf(fg, "gene%d\t%s\n", g + 1, gene_names[g]);
        else std::fprintf(fg, "gene%d\tgene%d\n", g + 1, g + 1);
    }
    const char* pre = barcode_prefix ? barcode_prefix : "cell";
    for (int64_t c = 0; c < N; ++c) std::fprintf(fb, "%s%lld\n", pre, (long long)(c + 1));
    const bool ok = std::fclose(fg) == 0 && std::fclose(fb) == 0;
    if (!ok) return fail(SCRNA_EINVAL, "cannot close genes.tsv / barcodes.tsv in %s", dir);
    return SCRNA_OK;
}
