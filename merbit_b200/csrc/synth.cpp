// Seeded synthetic CSR generators (declared in include/merbit_synth.h).
//
// The reference harness loads Matrix Market graphs by id
// (src/class.cu:60-141); none are available, so these generators produce the
// workloads instead.  Every row / edge / vector element draws from its own
// counter-based stream, so results do not depend on the OpenMP thread count.
//
// RNG: SplitMix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014) used as a counter hash: a stream is seeded by
// mixing (seed, tag, index) and then advanced by the golden-ratio increment.
#include "../../include/merbit_synth.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;

inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Stream {
    uint64_t s;
    Stream(uint64_t seed, uint64_t tag, uint64_t idx)
        : s(mix64(mix64(seed * kGolden + tag) ^ (idx * 0xD1B54A32D192ED03ull + kGolden))) {}
    uint64_t next() { return mix64(s += kGolden); }
    // uniform in [0,1) with 53 random bits
    double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
    // uniform in (0,1]
    double uniform_open0() { return ((double)(next() >> 11) + 1.0) * 0x1.0p-53; }
    // Box-Muller, one normal per call
    double normal() {
        double u1 = uniform_open0(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
    }
    // uniform integer in [0, n) (Lemire's multiply-shift; bias < n/2^64)
    int64_t below(int64_t n) {
        return (int64_t)(((unsigned __int128)next() * (unsigned __int128)(uint64_t)n) >> 64);
    }
};

enum : uint64_t {
    kTagZipfLen = 0x5a49504631ull,
    kTagZipfCol = 0x5a49504632ull,
    kTagZipfVal = 0x5a49504633ull,
    kTagStencil = 0x53544e4331ull,
    kTagRmatEdge = 0x524d415431ull,
    kTagRmatVal = 0x524d415432ull,
};

}  // namespace

extern "C" {

int merbit_synth_laplace2d(int64_t nx, int64_t ny, int32_t* row_ptr, int32_t* col, double* vals) {
    if (nx <= 0 || ny <= 0) return -1;
    const int64_t n = nx * ny;
    if (5 * n > INT32_MAX) return -2;
    // Row r = iy*nx + ix; its nonzero count is known in closed form, so
    // row_ptr is a prefix over rows computed per row in parallel.
    auto deg = [&](int64_t ix, int64_t iy) {
        return (int64_t)1 + (ix > 0) + (ix < nx - 1) + (iy > 0) + (iy < ny - 1);
    };
    // prefix: rows before (ix,iy) = full rows before iy + partial.
    std::vector<int64_t> rowstart(ny + 1, 0);
    for (int64_t iy = 0; iy < ny; ++iy) {
        int64_t s = 0;
        for (int64_t ix = 0; ix < nx; ++ix) s += deg(ix, iy);
        rowstart[iy + 1] = rowstart[iy] + s;
    }
#pragma omp parallel for schedule(static)
    for (int64_t iy = 0; iy < ny; ++iy) {
        int64_t e = rowstart[iy];
        for (int64_t ix = 0; ix < nx; ++ix) {
            const int64_t r = iy * nx + ix;
            row_ptr[r] = (int32_t)e;
            if (iy > 0) { col[e] = (int32_t)(r - nx); vals[e++] = -1.0; }
            if (ix > 0) { col[e] = (int32_t)(r - 1); vals[e++] = -1.0; }
            col[e] = (int32_t)r; vals[e++] = 4.0;
            if (ix < nx - 1) { col[e] = (int32_t)(r + 1); vals[e++] = -1.0; }
            if (iy < ny - 1) { col[e] = (int32_t)(r + nx); vals[e++] = -1.0; }
        }
    }
    row_ptr[n] = (int32_t)rowstart[ny];
    return 0;
}

int64_t merbit_synth_stencil27_nnz(int64_t nx, int64_t ny, int64_t nz) {
    if (nx <= 0 || ny <= 0 || nz <= 0) return -1;
    return (3 * nx - 2) * (3 * ny - 2) * (3 * nz - 2);
}

int merbit_synth_stencil27(int64_t nx, int64_t ny, int64_t nz, uint64_t seed, int32_t* row_ptr,
                           int32_t* col, double* vals) {
    const int64_t total = merbit_synth_stencil27_nnz(nx, ny, nz);
    if (total < 0) return -1;
    if (total > INT32_MAX) return -2;
    const int64_t plane = nx * ny, n = plane * nz;
    auto cnt1 = [](int64_t i, int64_t m) { return (int64_t)1 + (i > 0) + (i < m - 1); };
    // nonzeros of row (ix,iy,iz) = cnt(ix)*cnt(iy)*cnt(iz); prefix per z-plane
    // and per y-line is closed form, so each line is filled independently.
#pragma omp parallel for schedule(static) collapse(2)
    for (int64_t iz = 0; iz < nz; ++iz) {
        for (int64_t iy = 0; iy < ny; ++iy) {
            // nonzeros before plane iz: (3nx-2)(3ny-2) * (sum_{z<iz} cnt(z))
            int64_t zsum = 0;
            for (int64_t z = 0; z < iz; ++z) zsum += cnt1(z, nz);
            int64_t ysum = 0;
            for (int64_t y = 0; y < iy; ++y) ysum += cnt1(y, ny);
            int64_t e = (3 * nx - 2) * (3 * ny - 2) * zsum + (3 * nx - 2) * ysum * cnt1(iz, nz);
            for (int64_t ix = 0; ix < nx; ++ix) {
                const int64_t r = iz * plane + iy * nx + ix;
                row_ptr[r] = (int32_t)e;
                Stream st(seed, kTagStencil, (uint64_t)r);
                double off = 0.0;
                int64_t diag_pos = -1;
                for (int dz = -1; dz <= 1; ++dz) {
                    const int64_t z = iz + dz;
                    if (z < 0 || z >= nz) continue;
                    for (int dy = -1; dy <= 1; ++dy) {
                        const int64_t y = iy + dy;
                        if (y < 0 || y >= ny) continue;
                        for (int dx = -1; dx <= 1; ++dx) {
                            const int64_t x = ix + dx;
                            if (x < 0 || x >= nx) continue;
                            const int64_t c = z * plane + y * nx + x;
                            col[e] = (int32_t)c;
                            if (c == r) {
                                diag_pos = e;
                                vals[e] = 0.0;
                            } else {
                                const double v = st.normal();
                                vals[e] = v;
                                off += std::fabs(v);
                            }
                            ++e;
                        }
                    }
                }
                vals[diag_pos] = off + 1.0;
            }
        }
    }
    row_ptr[n] = (int32_t)total;
    return 0;
}

int64_t merbit_synth_zipf_rowptr(int64_t nrow, int64_t ncol, double s, int64_t cap,
                                 double empty_frac, uint64_t seed, int32_t* row_ptr) {
    if (nrow < 0 || ncol <= 0 || cap <= 0 || s <= 0.0) return -1;
    const int64_t kmax = std::min(cap, ncol);
    // CDF of P(L = k) proportional to k^-s on {1..kmax}.
    std::vector<double> cdf(kmax);
    double acc = 0.0;
    for (int64_t k = 1; k <= kmax; ++k) {
        acc += std::pow((double)k, -s);
        cdf[k - 1] = acc;
    }
    for (auto& c : cdf) c /= acc;
    std::vector<int64_t> len(nrow);
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nrow; ++r) {
        Stream st(seed, kTagZipfLen, (uint64_t)r);
        const double ue = st.uniform();
        const double ul = st.uniform();
        if (ue < empty_frac) {
            len[r] = 0;
        } else {
            int64_t k = std::upper_bound(cdf.begin(), cdf.end(), ul) - cdf.begin();
            len[r] = std::min(k + 1, kmax);
        }
    }
    int64_t tot = 0;
    for (int64_t r = 0; r < nrow; ++r) {
        if (tot > INT32_MAX) return -2;
        row_ptr[r] = (int32_t)tot;
        tot += len[r];
    }
    if (tot > INT32_MAX) return -2;
    row_ptr[nrow] = (int32_t)tot;
    return tot;
}

int merbit_synth_zipf_fill(int64_t nrow, int64_t ncol, uint64_t seed, const int32_t* row_ptr,
                           int32_t* col, double* vals) {
    if (nrow < 0 || ncol <= 0) return -1;
#pragma omp parallel
    {
        std::vector<int32_t> buf;
#pragma omp for schedule(dynamic, 64)
        for (int64_t r = 0; r < nrow; ++r) {
            const int64_t b = row_ptr[r], L = row_ptr[r + 1] - b;
            if (L <= 0) continue;
            Stream st(seed, kTagZipfCol, (uint64_t)r);
            int32_t* out = col + b;
            if (L * 4 >= ncol) {
                // selection sampling (Knuth, TAOCP vol. 2, Algorithm S): sorted, exact.
                int64_t need = L;
                for (int64_t i = 0; i < ncol && need > 0; ++i)
                    if ((double)(ncol - i) * st.uniform() < (double)need) {
                        *out++ = (int32_t)i;
                        --need;
                    }
            } else {
                buf.clear();
                while ((int64_t)buf.size() < L) {
                    const int64_t miss = L - (int64_t)buf.size();
                    for (int64_t i = 0; i < miss; ++i) buf.push_back((int32_t)st.below(ncol));
                    std::sort(buf.begin(), buf.end());
                    buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
                }
                std::memcpy(out, buf.data(), sizeof(int32_t) * (size_t)L);
            }
            Stream sv(seed, kTagZipfVal, (uint64_t)r);
            for (int64_t e = 0; e < L; ++e) vals[b + e] = sv.normal();
        }
    }
    return 0;
}

int64_t merbit_synth_rmat(int64_t n, int64_t nedges, double a, double b, double c, uint64_t seed,
                          int32_t* row_ptr, int32_t* col, double* vals) {
    if (n <= 0 || nedges < 0 || n > INT32_MAX) return -1;
    int scale = 0;
    while (((int64_t)1 << scale) < n) ++scale;
    // 1. every edge draws its (row, col) from its own stream
    std::vector<int32_t> er((size_t)nedges), ec((size_t)nedges);
    // Quadrant choice per level from u = uniform() in [0,1): row bit u >= a+b,
    // column bit a <= u < a+b or u >= a+b+c.  u is k * 2^-53 for the integer
    // k = next() >> 11, so each comparison u >= t equals k >= ceil(t * 2^53)
    // exactly; the integer form below draws the same bits without branches.
    auto threshold = [](double t) {
        const double s = std::ceil(t * 0x1.0p53);
        return s <= 0.0 ? 0ull : (s >= 0x1.0p53 ? (1ull << 53) : (uint64_t)s);
    };
    const uint64_t ta = threshold(a), tab = threshold(a + b), tabc = threshold(a + b + c);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nedges; ++e) {
        Stream st(seed, kTagRmatEdge, (uint64_t)e);
        uint64_t r, q;
        do {
            r = 0;
            q = 0;
            for (int l = 0; l < scale; ++l) {
                const uint64_t k = st.next() >> 11;
                const uint64_t rb = k >= tab;
                const uint64_t cb = ((k >= ta) & (k < tab)) | (k >= tabc);
                r = (r << 1) | rb;
                q = (q << 1) | cb;
            }
        } while ((int64_t)r >= n || (int64_t)q >= n);
        er[e] = (int32_t)r;
        ec[e] = (int32_t)q;
    }
    // 2. counting sort by row: per-chunk row histograms, then a scatter of
    // the columns into row buckets (O(edges), no comparison sort)
    const int nchunk = std::max(1, std::min(omp_get_max_threads(), 64));
    std::vector<int64_t> hist((size_t)nchunk * (size_t)n, 0);
    auto chunk_lo = [&](int t) { return nedges * t / nchunk; };
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nchunk; ++t) {
        int64_t* h = hist.data() + (size_t)t * n;
        for (int64_t e = chunk_lo(t); e < chunk_lo(t + 1); ++e) h[er[e]]++;
    }
    std::vector<int64_t> start((size_t)n + 1, 0);
    for (int64_t r = 0; r < n; ++r) {
        int64_t acc = start[r];
        for (int t = 0; t < nchunk; ++t) {
            const int64_t k = hist[(size_t)t * n + r];
            hist[(size_t)t * n + r] = acc;  // this chunk's first slot in row r
            acc += k;
        }
        start[r + 1] = acc;
    }
    std::vector<int32_t> bucket((size_t)nedges);
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nchunk; ++t) {
        int64_t* h = hist.data() + (size_t)t * n;
        for (int64_t e = chunk_lo(t); e < chunk_lo(t + 1); ++e) bucket[h[er[e]]++] = ec[e];
    }
    std::vector<int32_t>().swap(er);
    std::vector<int32_t>().swap(ec);
    std::vector<int64_t>().swap(hist);
    // 3. sort and de-duplicate the columns of each row
    std::vector<int64_t> ulen((size_t)n);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < n; ++r) {
        int32_t* lo = bucket.data() + start[r];
        int32_t* hi = bucket.data() + start[r + 1];
        std::sort(lo, hi);
        ulen[r] = std::unique(lo, hi) - lo;
    }
    int64_t nnz = 0;
    for (int64_t r = 0; r < n; ++r) {
        if (nnz > INT32_MAX) return -2;
        row_ptr[r] = (int32_t)nnz;
        nnz += ulen[r];
    }
    if (nnz > INT32_MAX) return -2;
    row_ptr[n] = (int32_t)nnz;
    // 4. compact into CSR; value e draws from stream e of the value tag
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < n; ++r) {
        std::memcpy(col + row_ptr[r], bucket.data() + start[r], sizeof(int32_t) * (size_t)ulen[r]);
        for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e) {
            Stream sv(seed, kTagRmatVal, (uint64_t)e);
            vals[e] = sv.normal();
        }
    }
    return nnz;
}

int merbit_synth_uniform(uint64_t seed, uint64_t tag, int64_t n, double lo, double hi, double* out) {
    if (n < 0) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        Stream st(seed, tag, (uint64_t)i);
        out[i] = lo + (hi - lo) * st.uniform();
    }
    return 0;
}

int merbit_synth_normal(uint64_t seed, uint64_t tag, int64_t n, double* out) {
    if (n < 0) return -1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        Stream st(seed, tag, (uint64_t)i);
        out[i] = st.normal();
    }
    return 0;
}

}  // extern "C"
