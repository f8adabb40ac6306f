// C ABI for the SpMM kernels (spmm.cu): one plan with k right-hand sides,
// and batches of plans run by one persistent launch.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "merbit_internal.cuh"

namespace merbit {

int alloc_spmm_slots(SpmmSlots* s, long long nslots, cudaStream_t st) {
    if (nslots <= 0) nslots = 1;
    if (nslots > INT_MAX) return fail(MERBIT_ERR_OVERFLOW, "spmm: tiles * k exceeds int32");
    const size_t words = 4 * (size_t)nslots;
    int rc = dev_alloc(&s->words, sizeof(unsigned long long) * words, st);
    if (rc == MERBIT_OK) rc = dev_alloc(&s->state, sizeof(LaunchState), st);
    if (rc != MERBIT_OK) {
        dev_free(s->words, st);
        s->words = nullptr;
        return rc;
    }
    MERBIT_CUDA(cudaMemsetAsync(s->words, 0xFF, sizeof(unsigned long long) * words, st));
    LaunchState init = {};
    init.epoch = 1u;
    MERBIT_CUDA(cudaMemcpyAsync(s->state, &init, sizeof(init), cudaMemcpyHostToDevice, st));
    MERBIT_CUDA(cudaStreamSynchronize(st));
    s->nslots = nslots;
    return MERBIT_OK;
}

namespace {

constexpr int kDefaultItems = 256;
constexpr int kBatchDefaultIpt = 11;
constexpr int kBatchDefaultVariant = 6;

bool pow2(int k) { return k > 0 && (k & (k - 1)) == 0; }

// Widest RHS vector per lane (4, 2, 1) that the leading dimension and the
// pointers allow for k columns of a type of `esz` bytes.
int pick_vw(int k, long long ldx, const void* x, const void* y, long long ldy, int esz,
            int items) {
    for (int vw = 4; vw >= 1; vw >>= 1) {
        if (vw > k || !spmm_config_exists(k, vw, items)) continue;
        if (vw == 1) return 1;
        const size_t a = (size_t)vw * esz;  // vector load size
        if (ldx % vw != 0) continue;
        if (((uintptr_t)x % (a < 16 ? a : 16)) != 0) continue;
        (void)y;
        (void)ldy;
        return vw;
    }
    return 1;
}

SpmmDesc make_desc(merbit_plan_s* p, const Partition* part, const void* x, long long ldx, void* y,
                   long long ldy, int tile_begin) {
    SpmmDesc d;
    d.row_ptr = p->row_ptr;
    d.col = p->col;
    d.vals = p->vals;
    d.x = x;
    d.y = y;
    d.ldx = ldx;
    d.ldy = ldy;
    d.coords = part->coords;
    d.nrow = p->nrow;
    d.nnz = p->nnz;
    d.num_tiles = part->num_tiles;
    d.tile_begin = tile_begin;
    d.ipt = 0;
    d.pad = 0;
    return d;
}

// One launch over columns [0, kk) of X / Y (pointers already offset).
int spmm_block(merbit_plan_s* p, int kk, double alpha, const void* x, long long ldx, double beta,
               void* y, long long ldy, cudaStream_t s, const void* dv_x = nullptr,
               long long dv_ldx = 0, void* dv_out = nullptr) {
    const int esz = (int)xy_size(p->dtype);
    // vector width: the widest the operands allow (with a fused dval, dv_x
    // rows are loaded with the same width)
    auto width = [&](int items) {
        int vw = pick_vw(kk, ldx, x, y, ldy, esz, items);
        if (dv_out)
            while (vw > 1 && (dv_ldx % vw != 0 || (uintptr_t)dv_x % ((size_t)vw * esz) != 0)) vw >>= 1;
        return vw;
    };
    // at vector width 4 (k >= 4) the larger tiles measured faster on the
    // power-law and banded matrices, and among them the one of an odd length
    // per lane group (480, 496, 504, 508 items at k = 4, 8, 16, 32: no bank
    // conflicts between the groups' segments; Zipf-1M at k = 16: 0.524 ms
    // against 0.570 at 512); other shapes keep 256
    int items = kDefaultItems;
    if (kk >= 4 && width(512) == 4) {
        items = 512;
        const int odd = spmm_odd_tile(kk);
        if (odd && width(odd) == 4) items = odd;
    }
    const int vw = width(items);
    if (!spmm_config_exists(kk, vw, items)) return MERBIT_ERR_UNSUPPORTED;
    const Partition* part = nullptr;
    int st = plan_partition(p, items, &part, s);
    if (st != MERBIT_OK) return st;
    const long long key = ((long long)kk << 20) | items;
    auto it = p->spmm_slots.find(key);
    if (it == p->spmm_slots.end()) {
        SpmmSlots sl;
        st = alloc_spmm_slots(&sl, (long long)part->num_tiles * kk, s);
        if (st != MERBIT_OK) return st;
        it = p->spmm_slots.emplace(key, sl).first;
    }
    SpmmLaunch a = {};
    a.single = make_desc(p, part, x, ldx, y, ldy, 0);
    a.descs = nullptr;
    a.ndesc = 0;
    a.nslots = (int)it->second.nslots;
    a.slots = it->second.words;
    a.xch = it->second.words + 2 * (size_t)it->second.nslots;
    a.state = it->second.state;
    a.total_tiles = part->num_tiles;
    a.alpha = alpha;
    a.beta = beta;
    if (dv_out) {
        a.dv_x = dv_x;
        a.dv_ldx = dv_ldx;
        a.dv_perm = p->perm;
        a.dv_out = dv_out;
    }
    return spmm_launch(p->dtype, kk, vw, items, a, s);
}

}  // namespace
}  // namespace merbit

// Batch of plans sharing one persistent launch.
struct merbit_batch_s {
    int count = 0, k = 0, dtype = 0, items = 256, vw = 1;
    // kernel 0: the SpMM kernel at vector width vw, matrix i with tiles of
    // tile[i] merge items, each `items` or (items2 != 0, vw = 4) `items2`;
    // kernel 1 (k = 1, 16-byte aligned arrays): the warp-tile kernel with
    // variant `variant` and ipt[i] items per lane for matrix i
    int kernel = 0, variant = 0, items2 = 0;
    std::vector<int> ipt, tile;
    bool all_vec = true;
    int device = 0;
    std::vector<merbit_plan_s*> plans;
    std::vector<const void*> x;
    std::vector<void*> y;
    std::vector<long long> ldx, ldy;
    merbit::SpmmDesc* d_descs = nullptr;
    int total_tiles = 0;
    merbit::SpmmSlots slots;
    double algorithmic_bytes = 0.0;
    long long nnz = 0;
};

using namespace merbit;

namespace {

// Uploads the descriptors and sizes the carry slots for `tot` tiles.
int batch_upload(merbit_batch_s* b, const std::vector<SpmmDesc>& h, long long tot, cudaStream_t s) {
    if (b->d_descs == nullptr) {
        int st = dev_alloc(&b->d_descs, sizeof(SpmmDesc) * b->count, s);
        if (st != MERBIT_OK) return st;
    }
    MERBIT_CUDA(cudaMemcpyAsync(b->d_descs, h.data(), sizeof(SpmmDesc) * b->count,
                                cudaMemcpyHostToDevice, s));
    if (b->slots.nslots < tot * b->k) {
        if (b->slots.words) MERBIT_CUDA(cudaDeviceSynchronize());  // launches may use them
        dev_free(b->slots.words, s);
        dev_free(b->slots.state, s);
        b->slots = SpmmSlots();
        int st = alloc_spmm_slots(&b->slots, tot * b->k, s);
        if (st != MERBIT_OK) return st;
    }
    MERBIT_CUDA(cudaStreamSynchronize(s));
    b->total_tiles = (int)tot;
    return MERBIT_OK;
}

// Widest vector width every member allows at `items` merge items per tile.
int batch_vw(const merbit_batch_s* b, int items) {
    int vw = 4;
    const int esz = (int)xy_size(b->dtype);
    for (int i = 0; i < b->count; ++i)
        vw = std::min(vw, pick_vw(b->k, b->ldx[i], b->x[i], b->y[i], b->ldy[i], esz, items));
    return spmm_config_exists(b->k, vw, items) ? vw : 1;
}

// The SpMM kernel, matrix i with tiles of tile[i] merge items (each `items`
// or `items2`; items2 = 0: `items` for every matrix).
int batch_build_tiles(merbit_batch_s* b, int items, int items2, const std::vector<int>& tile,
                      cudaStream_t s) {
    int vw = batch_vw(b, items);
    if (items2) {
        if (vw != 4 || batch_vw(b, items2) != 4 || !spmm_pair_exists(b->k, 4, items, items2))
            return fail(MERBIT_ERR_UNSUPPORTED,
                        "batch: no tile pair of these sizes for this k and these operands");
    }
    std::vector<SpmmDesc> h(b->count);
    long long tot = 0;
    for (int i = 0; i < b->count; ++i) {
        const int ti = items2 && tile[i] == items2 ? items2 : items;
        const Partition* part = nullptr;
        int st = plan_partition(b->plans[i], ti, &part, s);
        if (st != MERBIT_OK) return st;
        if (tot + part->num_tiles > INT_MAX) return fail(MERBIT_ERR_OVERFLOW, "batch: too many tiles");
        h[i] = make_desc(b->plans[i], part, b->x[i], b->ldx[i], b->y[i], b->ldy[i], (int)tot);
        h[i].ipt = ti;
        tot += part->num_tiles;
    }
    int st = batch_upload(b, h, tot, s);
    if (st != MERBIT_OK) return st;
    b->kernel = 0;
    b->items = items;
    b->items2 = items2;
    b->tile.assign(b->count, items);
    if (items2)
        for (int i = 0; i < b->count; ++i) b->tile[i] = tile[i] == items2 ? items2 : items;
    b->vw = vw;
    return MERBIT_OK;
}

// The SpMM kernel with `items` merge items per tile for every matrix.
int batch_build(merbit_batch_s* b, int items, cudaStream_t s) {
    return batch_build_tiles(b, items, 0, {}, s);
}

// The tile pair (smaller, larger) that `items` belongs to at k, or false.
bool tile_pair_of(int k, int items, int* lo, int* hi) {
    int c[8];
    const int n = spmm_tile_candidates(k, c);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (spmm_pair_exists(k, 4, c[i], c[j]) && (items == c[i] || items == c[j])) {
                *lo = c[i];
                *hi = c[j];
                return true;
            }
    return false;
}

// Nearest items per lane that `variant` takes.
int ipt_for_variant(int variant, int ipt) {
    return batch_variant_takes(variant, ipt) ? ipt : batch_variant_start_ipt(variant);
}

// The warp-tile kernel (k = 1) with b->ipt[i] items per lane for matrix i
// (items per lane the variant does not take become its starting value).
int batch_build_warp(merbit_batch_s* b, int variant, cudaStream_t s) {
    std::vector<SpmmDesc> h(b->count);
    long long tot = 0;
    for (int i = 0; i < b->count; ++i) {
        b->ipt[i] = ipt_for_variant(variant, b->ipt[i]);
        const Partition* part = nullptr;
        int st = plan_partition(b->plans[i], 32 * b->ipt[i], &part, s);
        if (st != MERBIT_OK) return st;
        if (tot + part->num_tiles > INT_MAX) return fail(MERBIT_ERR_OVERFLOW, "batch: too many tiles");
        h[i] = make_desc(b->plans[i], part, b->x[i], b->ldx[i], b->y[i], b->ldy[i], (int)tot);
        h[i].ipt = b->ipt[i];
        tot += part->num_tiles;
    }
    int st = batch_upload(b, h, tot, s);
    if (st != MERBIT_OK) return st;
    b->kernel = 1;
    b->variant = variant;
    b->items = 0;
    b->items2 = 0;
    b->tile.clear();
    b->vw = 1;
    return MERBIT_OK;
}

int batch_run(merbit_batch_s* b, double alpha, double beta, cudaStream_t s) {
    SpmmLaunch a = {};
    a.descs = b->d_descs;
    a.ndesc = b->count;
    a.nslots = (int)b->slots.nslots;
    a.slots = b->slots.words;
    a.xch = b->slots.words + 2 * (size_t)b->slots.nslots;
    a.state = b->slots.state;
    a.total_tiles = b->total_tiles;
    a.alpha = alpha;
    a.beta = beta;
    if (b->kernel == 1) return batch_warp_launch(b->dtype, b->variant, a, s);
    return spmm_launch(b->dtype, b->k, b->vw, b->items, a, s, b->items2);
}

// Mean ms of one batch launch (2 warm-up launches, then `reps` timed).
int time_batch(merbit_batch_s* b, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1, int reps,
               float* ms) {
    int st = MERBIT_OK;
    for (int w = 0; w < 2 && st == MERBIT_OK; ++w) st = batch_run(b, 1.0, 0.0, s);
    if (st != MERBIT_OK) return st;
    MERBIT_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps && st == MERBIT_OK; ++r) st = batch_run(b, 1.0, 0.0, s);
    if (st != MERBIT_OK) return st;
    MERBIT_CUDA(cudaEventRecord(e1, s));
    MERBIT_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    MERBIT_CUDA(cudaEventElapsedTime(&t, e0, e1));
    *ms = t / (float)reps;
    return MERBIT_OK;
}

int log2_floor(double v) {
    int b = 0;
    while (v >= 2.0 && b < 62) {
        v *= 0.5;
        ++b;
    }
    return b;
}

// Signature class of a batch member for the per-class search of the items
// per lane: mean row length and longest-row skew (both log2 buckets).
int batch_class(const merbit_plan_s* p) {
    const double mean = p->nrow > 0 ? (double)p->nnz / p->nrow : 0.0;
    const double skew = p->max_row_len > 0 ? (double)p->max_row_len / std::max(mean, 1.0) : 1.0;
    return log2_floor(mean + 1.0) * 64 + log2_floor(skew);
}

}  // namespace

extern "C" {

int merbit_spmm(merbit_plan plan, int32_t k, double alpha, const void* d_x, int64_t ldx,
                double beta, void* d_y, int64_t ldy, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "spmm: plan is null");
    if (k < 1) return fail(MERBIT_ERR_INVALID, "spmm: k < 1");
    if (ldx < k || ldy < k) return fail(MERBIT_ERR_INVALID, "spmm: leading dimension < k");
    if (plan->nrow == 0) return MERBIT_OK;
    if (!d_y || (plan->ncol > 0 && !d_x)) return fail(MERBIT_ERR_INVALID, "spmm: X/Y is null");
    cudaStream_t s = (cudaStream_t)stream;
    const size_t esz = xy_size(plan->dtype);
    // power-of-two column blocks of at most 32
    int j = 0;
    while (j < k) {
        int kk = 32;
        while (kk > k - j) kk >>= 1;
        const char* xb = static_cast<const char*>(d_x) + (size_t)j * esz;
        char* yb = static_cast<char*>(d_y) + (size_t)j * esz;
        int st = spmm_block(plan, kk, alpha, xb, ldx, beta, yb, ldy, s);
        if (st != MERBIT_OK) return st;
        j += kk;
    }
    return MERBIT_OK;
}

int merbit_spmm_dval(merbit_plan tplan, int32_t k, const void* d_g, int64_t ldg, const void* d_x,
                     int64_t ldx, void* d_dx, int64_t lddx, void* d_dval, void* stream) {
    if (!tplan) return fail(MERBIT_ERR_INVALID, "spmm_dval: plan is null");
    if (!tplan->perm) return fail(MERBIT_ERR_INVALID, "spmm_dval: not a transpose plan");
    if (k < 1 || ldg < k || ldx < k || lddx < k)
        return fail(MERBIT_ERR_INVALID, "spmm_dval: bad k / leading dimension");
    if (tplan->dtype == MERBIT_BF16)
        return fail(MERBIT_ERR_UNSUPPORTED, "spmm_dval: bf16 values (use merbit_spmm + merbit_dval)");
    if (!pow2(k) || k > 32)
        return fail(MERBIT_ERR_UNSUPPORTED, "spmm_dval: k must be 1, 2, 4, 8, 16 or 32");
    if (tplan->nrow == 0) return MERBIT_OK;
    if (!d_dx || !d_dval || (tplan->ncol > 0 && !d_g) || !d_x)
        return fail(MERBIT_ERR_INVALID, "spmm_dval: null pointer");
    const int st = spmm_block(tplan, k, 1.0, d_g, ldg, 0.0, d_dx, lddx, (cudaStream_t)stream, d_x,
                              ldx, d_dval);
    if (st == MERBIT_ERR_UNSUPPORTED)
        return fail(MERBIT_ERR_UNSUPPORTED, "spmm_dval: no configuration for these operands");
    return st;
}

int merbit_batch_create(merbit_batch* batch, int32_t count, const merbit_plan* plans, int32_t k,
                        const void* const* d_x, const int64_t* ldx, void* const* d_y,
                        const int64_t* ldy, void* stream) {
    if (!batch) return fail(MERBIT_ERR_INVALID, "batch_create: batch is null");
    *batch = nullptr;
    if (count < 1 || !plans || !d_x || !d_y || !ldx || !ldy)
        return fail(MERBIT_ERR_INVALID, "batch_create: bad arguments");
    if (!pow2(k) || k > 32) return fail(MERBIT_ERR_UNSUPPORTED, "batch_create: k must be 1, 2, 4, 8, 16 or 32");
    auto* b = new merbit_batch_s();
    cudaGetDevice(&b->device);
    b->count = count;
    b->k = k;
    b->dtype = plans[0] ? plans[0]->dtype : 0;
    for (int i = 0; i < count; ++i) {
        merbit_plan_s* p = plans[i];
        if (!p || p->dtype != b->dtype || ldx[i] < k || ldy[i] < k ||
            (p->nrow > 0 && !d_y[i]) || (p->ncol > 0 && !d_x[i])) {
            delete b;
            return fail(MERBIT_ERR_INVALID, "batch_create: plan " + std::to_string(i) +
                                                " is null, of another dtype, or has bad X/Y");
        }
        b->plans.push_back(p);
        b->all_vec = b->all_vec && p->vec;
        b->x.push_back(d_x[i]);
        b->y.push_back(d_y[i]);
        b->ldx.push_back(ldx[i]);
        b->ldy.push_back(ldy[i]);
        b->nnz += p->nnz;
        b->algorithmic_bytes += 4.0 * (p->nrow + 1.0) + (double)p->nnz * (4.0 + (double)dtype_size(p->dtype)) +
                                (double)k * (double)xy_size(p->dtype) * ((double)p->ncol + p->nrow);
    }
    // k = 1 on 16-byte aligned arrays: the warp-tile kernel in the variant
    // that measured fastest on the R-MAT batch (58% carveout, stages for 11
    // items per lane), each matrix starting from the items per lane cached
    // for its signature
    // (and the variant they were tuned in, when every cached member agrees)
    int st;
    if (k == 1 && b->all_vec) {
        int variant = -1;
        bool agree = true;
        for (auto* p : b->plans) {
            int v = -1;
            const int c = tune_cache_batch_ipt(p, &v);
            b->ipt.push_back(c > 0 ? c : kBatchDefaultIpt);
            if (v >= 0) {
                agree = agree && (variant < 0 || variant == v);
                variant = v;
            }
        }
        if (variant < 0 || !agree) variant = kBatchDefaultVariant;
        st = batch_build_warp(b, variant, (cudaStream_t)stream);
    } else {
        if (k == 1) b->ipt.assign(count, kBatchDefaultIpt);
        // untuned SpMM batches start from the tile the tuner picked on the
        // 128-matrix R-MAT batch: at vector width 4 the odd tile of k (480,
        // 496, 504, 508 items at k = 4, 8, 16, 32; 2.38 against 3.24 ms at
        // k = 4 for 256), at k = 2 the staged products in 352-item tiles
        // (2.10 against 2.85 ms), else 256
        int items = kDefaultItems;
        if (k >= 4) {
            const int odd = spmm_odd_tile(k);
            if (odd && batch_vw(b, odd) == 4) items = odd;
        } else if (k == 2 && batch_vw(b, 352) == 2) {
            items = 352;
        }
        st = batch_build(b, items, (cudaStream_t)stream);
    }
    if (st != MERBIT_OK) {
        merbit_batch_destroy(b);
        return st;
    }
    *batch = b;
    return MERBIT_OK;
}

int merbit_batch_spmm(merbit_batch batch, double alpha, double beta, void* stream) {
    if (!batch) return fail(MERBIT_ERR_INVALID, "batch_spmm: batch is null");
    return batch_run(batch, alpha, beta, (cudaStream_t)stream);
}

int merbit_batch_tune(merbit_batch batch, void* stream) {
    if (!batch) return fail(MERBIT_ERR_INVALID, "batch_tune: batch is null");
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    MERBIT_CUDA(cudaEventCreate(&e0));
    MERBIT_CUDA(cudaEventCreate(&e1));
    int st = MERBIT_OK;
    // 1. the kernel: the SpMM kernel at each tile size and vector width,
    //    and (k = 1, aligned arrays) the warp-tile kernel in each variant
    //    with the current items per lane
    int best_kernel = batch->kernel, best_items = batch->items, best_vw = batch->vw;
    int best_variant = batch->variant;
    float best = 1e30f;
    // candidates of this step: (ms, kernel, items or variant, vector width)
    std::vector<std::tuple<float, int, int, int>> cands;
    int items_c[8];
    const int nitems = spmm_tile_candidates(batch->k, items_c);
    for (int ii = 0; ii < nitems && st == MERBIT_OK; ++ii) {
        st = batch_build(batch, items_c[ii], s);
        if (st != MERBIT_OK) break;
        const int vmax = batch->vw;
        for (int vw = vmax; vw >= 1 && st == MERBIT_OK; vw >>= 1) {
            if (!spmm_config_exists(batch->k, vw, items_c[ii])) continue;
            batch->vw = vw;
            float ms = 0.f;
            st = time_batch(batch, s, e0, e1, 3, &ms);
            if (st == MERBIT_OK) cands.emplace_back(ms, 0, items_c[ii], vw);
        }
    }
    // the warp-tile kernel's variants, every matrix at the variant's
    // starting items per lane
    const bool warp_ok = batch->k == 1 && batch->all_vec;
    for (int v = 0; warp_ok && v < kBatchWarpVariants && st == MERBIT_OK; ++v) {
        batch->ipt.assign(batch->count, batch_variant_start_ipt(v));
        st = batch_build_warp(batch, v, s);
        float ms = 0.f;
        if (st == MERBIT_OK) st = time_batch(batch, s, e0, e1, 3, &ms);
        if (st == MERBIT_OK) cands.emplace_back(ms, 1, v, 1);
    }
    // the three fastest again, best of two rounds of 8 launches each (one
    // round of 3 cannot separate entries within a few percent)
    if (st == MERBIT_OK && !cands.empty()) {
        std::stable_sort(cands.begin(), cands.end(),
                         [](const auto& a, const auto& b) { return std::get<0>(a) < std::get<0>(b); });
        const size_t top = std::min<size_t>(3, cands.size());
        for (int round = 0; round < 2 && st == MERBIT_OK; ++round)
            for (size_t i = 0; i < top && st == MERBIT_OK; ++i) {
                const int kern = std::get<1>(cands[i]), opt = std::get<2>(cands[i]);
                if (kern == 0) {
                    st = batch_build(batch, opt, s);
                    batch->vw = std::get<3>(cands[i]);
                } else {
                    batch->ipt.assign(batch->count, batch_variant_start_ipt(opt));
                    st = batch_build_warp(batch, opt, s);
                }
                float ms = 0.f;
                if (st == MERBIT_OK) st = time_batch(batch, s, e0, e1, 8, &ms);
                if (st == MERBIT_OK && ms < best) {
                    best = ms;
                    best_kernel = kern;
                    if (kern == 0) {
                        best_items = opt;
                        best_vw = std::get<3>(cands[i]);
                    } else {
                        best_variant = opt;
                    }
                }
            }
    }
    if (warp_ok) batch->ipt.assign(batch->count, batch_variant_start_ipt(best_variant));
    // 2. warp-tile kernel: the items per lane per signature class, largest
    //    classes first, one pass of coordinate descent over the classes
    if (st == MERBIT_OK && best_kernel == 1) {
        std::map<int, long long> class_nnz;
        for (auto* p : batch->plans) class_nnz[batch_class(p)] += p->nnz;
        std::vector<std::pair<long long, int>> order;
        for (auto& kv : class_nnz) order.push_back({-kv.second, kv.first});
        std::sort(order.begin(), order.end());
        for (auto& oc : order) {
            const int cls = oc.second;
            std::vector<int> keep = batch->ipt;
            int best_ipt = -1;
            for (int c = 0; c < kNumBatchIpts && st == MERBIT_OK; ++c) {
                if (!batch_variant_takes(best_variant, kBatchIpts[c])) continue;
                for (int i = 0; i < batch->count; ++i)
                    if (batch_class(batch->plans[i]) == cls) batch->ipt[i] = kBatchIpts[c];
                st = batch_build_warp(batch, best_variant, s);
                float ms = 0.f;
                if (st == MERBIT_OK) st = time_batch(batch, s, e0, e1, 8, &ms);
                if (st == MERBIT_OK && ms < best) {
                    best = ms;
                    best_ipt = kBatchIpts[c];
                }
            }
            if (st != MERBIT_OK) break;
            batch->ipt = keep;
            if (best_ipt > 0)
                for (int i = 0; i < batch->count; ++i)
                    if (batch_class(batch->plans[i]) == cls) batch->ipt[i] = best_ipt;
        }
        if (st == MERBIT_OK)
            for (int i = 0; i < batch->count; ++i)
                tune_cache_store_batch_ipt(batch->plans[i], best_variant, batch->ipt[i]);
    }
    // 3. SpMM kernel at vector width 4: the tile size per signature class,
    //    between the two of the winning size's pair, one pass of coordinate
    //    descent over the classes
    int lo = 0, hi = 0;
    std::vector<int> best_tile(batch->count, best_items);
    bool paired = false;
    if (st == MERBIT_OK && best_kernel == 0 && best_vw == 4 &&
        tile_pair_of(batch->k, best_items, &lo, &hi)) {
        std::map<int, long long> class_nnz;
        for (auto* p : batch->plans) class_nnz[batch_class(p)] += p->nnz;
        std::vector<std::pair<long long, int>> order;
        for (auto& kv : class_nnz) order.push_back({-kv.second, kv.first});
        std::sort(order.begin(), order.end());
        std::vector<int> cur = best_tile;
        for (auto& oc : order) {
            const int cls = oc.second;
            std::vector<int> trial = cur;
            const int other = best_items == lo ? hi : lo;
            bool any = false;
            for (int i = 0; i < batch->count; ++i)
                if (batch_class(batch->plans[i]) == cls && trial[i] != other) {
                    trial[i] = other;
                    any = true;
                }
            if (!any) continue;
            st = batch_build_tiles(batch, lo, hi, trial, s);
            if (st == MERBIT_ERR_UNSUPPORTED) {
                st = MERBIT_OK;  // the operands take no pair
                break;
            }
            float ms = 0.f;
            if (st == MERBIT_OK) st = time_batch(batch, s, e0, e1, 8, &ms);
            if (st != MERBIT_OK) break;
            if (ms < best) {
                best = ms;
                cur = trial;
                paired = true;
            }
        }
        best_tile = cur;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MERBIT_OK) return st;
    if (best_kernel == 1) return batch_build_warp(batch, best_variant, s);
    st = paired ? batch_build_tiles(batch, lo, hi, best_tile, s) : batch_build(batch, best_items, s);
    if (st != MERBIT_OK) return st;
    batch->vw = best_vw;
    return MERBIT_OK;
}

int merbit_batch_set_kernel(merbit_batch batch, int32_t kernel, int32_t option, void* stream) {
    if (!batch) return fail(MERBIT_ERR_INVALID, "batch_set_kernel: batch is null");
    cudaStream_t s = (cudaStream_t)stream;
    if (kernel == 0) {
        int cand[8];
        const int n = spmm_tile_candidates(batch->k, cand);
        bool known = false;
        for (int i = 0; i < n; ++i) known = known || cand[i] == option;
        if (!known)
            return fail(MERBIT_ERR_INVALID, "batch_set_kernel: no SpMM tile of that size for this k");
        return batch_build(batch, option, s);
    }
    if (kernel == 1) {
        if (batch->k != 1 || !batch->all_vec)
            return fail(MERBIT_ERR_UNSUPPORTED,
                        "batch_set_kernel: the warp-tile kernel needs k = 1 and 16-byte aligned arrays");
        if (option < 0 || option >= kBatchWarpVariants)
            return fail(MERBIT_ERR_INVALID, "batch_set_kernel: no such variant");
        return batch_build_warp(batch, option, s);
    }
    return fail(MERBIT_ERR_INVALID, "batch_set_kernel: kernel is 0 or 1");
}

int merbit_batch_set_matrix_config(merbit_batch batch, int32_t index, int32_t items_per_thread,
                                   void* stream) {
    if (!batch) return fail(MERBIT_ERR_INVALID, "batch_set_matrix_config: batch is null");
    if (index < 0 || index >= batch->count)
        return fail(MERBIT_ERR_INVALID, "batch_set_matrix_config: index out of range");
    if (batch->k != 1 || !batch->all_vec)
        return fail(MERBIT_ERR_UNSUPPORTED,
                    "batch_set_matrix_config: per-matrix tiles need k = 1 and 16-byte aligned arrays");
    const int variant = batch->kernel == 1 ? batch->variant : 0;
    if (!batch_variant_takes(variant, items_per_thread))
        return fail(MERBIT_ERR_INVALID,
                    "batch_set_matrix_config: the kernel variant in use does not take that many "
                    "items per lane (variants 0-2 and 5: 7, 11, 15; 3-4: 15, 19, 23; 6-9: 7, 11); "
                    "select the variant first with merbit_batch_set_kernel");
    batch->ipt[index] = items_per_thread;
    return batch_build_warp(batch, variant, (cudaStream_t)stream);
}

int merbit_batch_set_matrix_tile(merbit_batch batch, int32_t index, int32_t tile_items,
                                 void* stream) {
    if (!batch) return fail(MERBIT_ERR_INVALID, "batch_set_matrix_tile: batch is null");
    if (index < 0 || index >= batch->count)
        return fail(MERBIT_ERR_INVALID, "batch_set_matrix_tile: index out of range");
    if (batch->kernel != 0)
        return fail(MERBIT_ERR_UNSUPPORTED,
                    "batch_set_matrix_tile: the batch runs the warp-tile kernel (use "
                    "merbit_batch_set_matrix_config, or merbit_batch_set_kernel(0, ...) first)");
    int lo = 0, hi = 0;
    if (batch->vw != 4 || !tile_pair_of(batch->k, batch->items, &lo, &hi) ||
        (tile_items != lo && tile_items != hi))
        return fail(MERBIT_ERR_INVALID,
                    "batch_set_matrix_tile: at vector width 4, k = 4, 8, 16 or 32, a matrix may "
                    "take the other tile of the batch's pair (256/512, or the two odd tiles of k)");
    std::vector<int> tile = batch->tile;
    tile[index] = tile_items;
    bool uniform = true;
    for (int t : tile) uniform = uniform && t == tile[0];
    if (uniform) return batch_build(batch, tile[0], (cudaStream_t)stream);
    return batch_build_tiles(batch, lo, hi, tile, (cudaStream_t)stream);
}

int merbit_batch_get_matrix_config(merbit_batch batch, int32_t index, int32_t* kernel,
                                   int32_t* tile_items, int32_t* items_per_thread) {
    if (!batch || !kernel || !tile_items || !items_per_thread)
        return fail(MERBIT_ERR_INVALID, "batch_get_matrix_config: null pointer");
    if (index < 0 || index >= batch->count)
        return fail(MERBIT_ERR_INVALID, "batch_get_matrix_config: index out of range");
    *kernel = batch->kernel;
    if (batch->kernel == 1) {
        *items_per_thread = batch->ipt[index];
        *tile_items = 32 * batch->ipt[index];
    } else {
        *tile_items = batch->tile.empty() ? batch->items : batch->tile[index];
        *items_per_thread = *tile_items / 32;
    }
    return MERBIT_OK;
}

int merbit_batch_get_info(merbit_batch batch, merbit_batch_info* info) {
    if (!batch || !info) return fail(MERBIT_ERR_INVALID, "batch_get_info: null pointer");
    info->count = batch->count;
    info->k = batch->k;
    info->dtype = batch->dtype;
    info->tile_items = batch->items;
    info->vector_width = batch->vw;
    info->total_tiles = batch->total_tiles;
    info->nnz = batch->nnz;
    info->algorithmic_bytes = batch->algorithmic_bytes;
    info->kernel = batch->kernel;
    info->variant = batch->variant;
    return MERBIT_OK;
}

int merbit_batch_destroy(merbit_batch batch) {
    if (!batch) return MERBIT_OK;
    // wait for the batch's launches, as cudaFree does, then release
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != batch->device) cudaSetDevice(batch->device);
    cudaDeviceSynchronize();
    dev_free(batch->d_descs, nullptr);
    dev_free(batch->slots.words, nullptr);
    dev_free(batch->slots.state, nullptr);
    if (cur != batch->device) cudaSetDevice(cur);
    delete batch;
    return MERBIT_OK;
}

}  // extern "C"
