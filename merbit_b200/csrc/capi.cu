// C ABI: plan lifetime, SpMV dispatch, tuning, error reporting.
//
// The plan plays the part of the reference's per-call setup in Fun_Merbit
// (include/tile.cuh:563-615: offset build, TILE construction, y/z buffers),
// done once and reused: the partition for the chosen tile size and the
// carry slots stay resident in HBM across launches.
#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>

#include "merbit_internal.cuh"

namespace merbit {

namespace {
thread_local std::string g_detail;
thread_local int g_last_cuda = 0;
}  // namespace

void set_error_detail(const std::string& s) { g_detail = s; }

int fail(int status, const std::string& detail) {
    g_detail = detail;
    return status;
}

int cuda_fail(cudaError_t e, const char* where) {
    g_last_cuda = (int)e;
    g_detail = std::string(where) + ": " + cudaGetErrorString(e);
    // un-latch a non-sticky error so that a later launch check of this
    // thread does not report it again (a sticky error stays)
    cudaGetLastError();
    return MERBIT_ERR_CUDA;
}


namespace {

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Grows the plan's carry slots to `tiles` (both parity arrays start empty:
// all ones).  The fill is ordered on s; callers synchronize s before a
// launch on another stream can use the slots.
int grow_carry(merbit_plan_s* p, int tiles, cudaStream_t s) {
    if (tiles <= p->slots) return MERBIT_OK;
    if (p->carry) {  // launches in flight may still use the old slots
        MERBIT_CUDA(cudaDeviceSynchronize());
        dev_free(p->carry, s);
        p->carry = nullptr;
        p->slots = 0;
    }
    const size_t words = 4 * (size_t)tiles;  // carries + boundary swaps, 2 parities
    int st = dev_alloc(&p->carry, sizeof(unsigned long long) * words, s);
    if (st != MERBIT_OK) return st;
    MERBIT_CUDA(cudaMemsetAsync(p->carry, 0xFF, sizeof(unsigned long long) * words, s));
    p->slots = tiles;
    return MERBIT_OK;
}

// Starts a partition for `tile_items` without synchronizing; its largest
// rows-per-tile lands in p->scratch->max_rows for the caller's next
// readback.  On failure nothing is added to the plan.
int plan_partition_start(merbit_plan_s* p, int tile_items, Partition** out, cudaStream_t s) {
    MERBIT_CUDA(cudaMemsetAsync(&p->scratch->max_rows, 0, sizeof(int), s));
    Partition q;
    int st = build_partition_async(p->row_ptr, p->nrow, p->nnz, tile_items, &q,
                                   &p->scratch->max_rows, s);
    if (st == MERBIT_OK) st = grow_carry(p, q.num_tiles, s);
    if (st != MERBIT_OK) {
        dev_free(q.coords, s);
        return st;
    }
    p->parts.push_back(q);
    *out = &p->parts.back();
    return MERBIT_OK;
}

}  // namespace

// Ensures the plan holds a partition for `tile_items` and enough carry
// slots; returns it in *out.  Synchronizes s when it builds one.
int plan_partition(merbit_plan_s* p, int tile_items, const Partition** out, cudaStream_t s) {
    for (auto& q : p->parts)
        if (q.tile_items == tile_items) {
            *out = &q;
            return MERBIT_OK;
        }
    Partition* q = nullptr;
    int st = plan_partition_start(p, tile_items, &q, s);
    if (st != MERBIT_OK) return st;
    int h_max = 0;
    cudaError_t e = cudaMemcpyAsync(&h_max, &p->scratch->max_rows, sizeof(int),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dev_free(q->coords, s);
        p->parts.pop_back();
        return cuda_fail(e, "partition: max rows");
    }
    q->max_rows = h_max;
    *out = q;
    return MERBIT_OK;
}

namespace {

// Whether configuration idx can run this plan (builds its partition).
int plan_config_ok(merbit_plan_s* p, int idx, bool* ok, cudaStream_t s) {
    *ok = false;
    const SpmvConfig c = spmv_config(p->dtype, idx);
    if (!spmv_config_allowed(c, p->vec)) return MERBIT_OK;
    if (c.kind == 3) {  // row groups: no partition, any matrix
        *ok = true;
        return MERBIT_OK;
    }
    const Partition* part = nullptr;
    int st = plan_partition(p, spmv_tile_items(c), &part, s);
    if (st != MERBIT_OK) return st;
    *ok = part->max_rows <= spmv_config_row_cap(c);
    return MERBIT_OK;
}

// First usable configuration in table order.
int plan_pick_default(merbit_plan_s* p, cudaStream_t s) {
    const int n = spmv_num_configs(p->dtype);
    for (int i = 0; i < n; ++i) {
        bool ok = false;
        int st = plan_config_ok(p, i, &ok, s);
        if (st != MERBIT_OK) return st;
        if (ok) {
            p->cfg = i;
            return MERBIT_OK;
        }
    }
    return fail(MERBIT_ERR_UNSUPPORTED, "no SpMV configuration fits this matrix");
}

// Grows the plan's residual partials to hold one word per CTA of any launch
// over `num_tiles` tiles (warp-tile kernel: at most 32 resident CTAs per SM;
// CTA-tile kernel: one CTA per tile).
int plan_partials(merbit_plan_s* p, int num_tiles, cudaStream_t s) {
    int sms = 0;
    MERBIT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device));
    const long long need = std::max<long long>(num_tiles, 32LL * std::max(sms, 1));
    if (need <= p->npartials) return MERBIT_OK;
    dev_free(p->partials, s);  // ordered after this plan's earlier launches
    p->partials = nullptr;
    p->npartials = 0;
    int st = dev_alloc(&p->partials, sizeof(double) * (size_t)need, s);
    if (st != MERBIT_OK) return st;
    p->npartials = need;
    return MERBIT_OK;
}

// y = alpha A x + beta z (z NULL: y); residual != NULL also writes
// *residual = sum_r |y[r] - x[r]| from the same launch.
int run_spmv(merbit_plan_s* p, int cfg, double alpha, const void* x, double beta, void* y,
             cudaStream_t s, const void* z = nullptr, double* residual = nullptr) {
    const SpmvConfig c = spmv_config(p->dtype, cfg);
    const Partition* part = nullptr;
    int st = MERBIT_OK;
    if (c.kind != 3) {
        st = plan_partition(p, spmv_tile_items(c), &part, s);
        if (st != MERBIT_OK) return st;
    }
    if (residual) {
        st = plan_partials(p, part ? part->num_tiles : 0, s);
        if (st != MERBIT_OK) return st;
    }
    SpmvLaunch a;
    a.row_ptr = p->row_ptr;
    a.col = p->col;
    a.vals = p->vals;
    a.x = x;
    a.y = y;
    a.coords = part ? part->coords : nullptr;
    a.slots = p->carry;
    a.xch = p->carry + 2 * (size_t)p->slots;
    a.nslots = p->slots;
    a.state = p->state;
    a.nrow = p->nrow;
    a.nnz = p->nnz;
    a.num_tiles = part ? part->num_tiles : 0;
    a.alpha = alpha;
    a.beta = beta;
    a.z = z;
    if (residual) {
        a.xres = x;
        a.partials = p->partials;
        a.residual = residual;
    }
    return spmv_launch(p->dtype, cfg, p->vec, a, s);
}

// Tuning cache: matrix signature -> config index.  The signature buckets
// (log2) the row count, the nonzero count, the density and the longest row,
// so that a configuration tuned on short, even rows (a stencil, where the
// row-group kernel wins) is never applied to a power-law matrix of the same
// size, whose long rows serialize that kernel.
struct Sig {
    int dtype, vec, nrow_bucket, nnz_bucket, density_bucket, maxrow_bucket;
    auto key() const {
        return std::tie(dtype, vec, nrow_bucket, nnz_bucket, density_bucket, maxrow_bucket);
    }
    bool operator<(const Sig& o) const { return key() < o.key(); }
    bool same_size(const Sig& o) const {
        return std::tie(dtype, vec, nrow_bucket, nnz_bucket, density_bucket) ==
               std::tie(o.dtype, o.vec, o.nrow_bucket, o.nnz_bucket, o.density_bucket);
    }
};
struct Tuned {
    int cfg;          // the configuration that won
    int max_row_len;  // longest row of the matrix it was tuned on
};
std::mutex g_tune_mu;
std::map<Sig, Tuned> g_tune;

int log2_bucket(double v) {
    int b = 0;
    while (v >= 2.0 && b < 62) {
        v *= 0.5;
        ++b;
    }
    return b;
}

Sig signature(const merbit_plan_s* p, int max_row_len) {
    Sig s;
    s.dtype = p->dtype;
    s.vec = p->vec;
    s.nrow_bucket = log2_bucket((double)p->nrow);
    s.nnz_bucket = log2_bucket((double)p->nnz);
    s.density_bucket = log2_bucket(4.0 * (double)p->nnz / (double)(p->nrow > 0 ? p->nrow : 1));
    s.maxrow_bucket = log2_bucket((double)(max_row_len > 0 ? max_row_len : 0) + 1.0);
    return s;
}

// Whether a cached choice may serve a plan whose longest row is
// max_row_len.  The row-group kernel gives each row to one lane group, so
// its time grows with the longest row: it is kept only for matrices whose
// longest row is at most twice the one it was tuned on.  Merge-path
// kernels balance any row lengths and are checked by their rows-per-tile
// cap instead.
bool cached_choice_fits(int dtype, const Tuned& t, int max_row_len) {
    if (spmv_config(dtype, t.cfg).kind != 3) return true;
    return (long long)max_row_len <= 2LL * std::max(t.max_row_len, 1);
}

// Batched k = 1 warp-tile kernel: the (variant, items per lane) the batch
// tuner chose for a matrix signature (same signature as the SpMV tuner's).
std::map<Sig, std::pair<int, int>> g_batch_ipt;

}  // namespace

int tune_cache_batch_ipt(const merbit_plan_s* p, int* variant) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const Sig sg = signature(p, p->max_row_len);
    *variant = -1;
    auto it = g_batch_ipt.find(sg);
    if (it != g_batch_ipt.end()) {
        *variant = it->second.first;
        return it->second.second;
    }
    // a warp-tile SpMV configuration tuned for this signature suggests its
    // items per lane when the batch kernel has the same
    auto jt = g_tune.find(sg);
    if (jt != g_tune.end()) {
        const SpmvConfig c = spmv_config(p->dtype, jt->second.cfg);
        if (c.kind == 1)
            for (int i = 0; i < kNumBatchIpts; ++i)
                if (kBatchIpts[i] == c.ipt) return c.ipt;
    }
    return -1;
}

void tune_cache_store_batch_ipt(const merbit_plan_s* p, int variant, int ipt) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_batch_ipt[signature(p, p->max_row_len)] = {variant, ipt};
}

}  // namespace merbit

using namespace merbit;

extern "C" {

const char* merbit_status_string(int status) {
    switch (status) {
    case MERBIT_OK: return "MERBIT_OK";
    case MERBIT_ERR_INVALID: return "MERBIT_ERR_INVALID: invalid argument";
    case MERBIT_ERR_MATRIX: return "MERBIT_ERR_MATRIX: malformed CSR structure";
    case MERBIT_ERR_OVERFLOW: return "MERBIT_ERR_OVERFLOW: nrow+nnz exceeds the int32 range";
    case MERBIT_ERR_CUDA: return "MERBIT_ERR_CUDA: CUDA runtime error";
    case MERBIT_ERR_TIMEOUT: return "MERBIT_ERR_TIMEOUT: device-side carry wait ran out";
    case MERBIT_ERR_UNSUPPORTED: return "MERBIT_ERR_UNSUPPORTED: not implemented";
    default: return "MERBIT: unknown status";
    }
}

int merbit_last_cuda_error(void) { return g_last_cuda; }

const char* merbit_last_error_detail(void) { return g_detail.c_str(); }

int merbit_plan_create(merbit_plan* plan, int32_t nrow, int32_t ncol, int32_t nnz,
                       const int32_t* d_row_ptr, const int32_t* d_col_idx, const void* d_vals,
                       merbit_dtype dtype, uint32_t flags, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "plan_create: plan is null");
    *plan = nullptr;
    if (nrow < 0 || ncol < 0 || nnz < 0) return fail(MERBIT_ERR_INVALID, "plan_create: negative size");
    if (dtype != MERBIT_F64 && dtype != MERBIT_F32 && dtype != MERBIT_BF16)
        return fail(MERBIT_ERR_INVALID, "plan_create: unknown dtype");
    if (!d_row_ptr) return fail(MERBIT_ERR_INVALID, "plan_create: row_ptr is null");
    if (nnz > 0 && (!d_col_idx || !d_vals))
        return fail(MERBIT_ERR_INVALID, "plan_create: col_idx/vals null with nnz > 0");
    if (nnz > 0 && ncol == 0) return fail(MERBIT_ERR_MATRIX, "plan_create: nnz > 0 with ncol == 0");
    if ((long long)nrow + nnz > (long long)INT_MAX - 64)
        return fail(MERBIT_ERR_OVERFLOW, "plan_create: nrow+nnz exceeds the int32 merge-path range");
    cudaStream_t s = (cudaStream_t)stream;
    auto* p = new merbit_plan_s();
    p->nrow = nrow;
    p->ncol = ncol;
    p->nnz = nnz;
    p->dtype = dtype;
    p->row_ptr = d_row_ptr;
    p->col = d_col_idx;
    p->vals = d_vals;
    p->vec = aligned16(d_col_idx) && aligned16(d_vals) && aligned16(d_row_ptr);
    cudaGetDevice(&p->device);
    // A provisional choice before the longest row is known: a cached
    // configuration of a matrix of the same size class (any longest-row
    // bucket; the exact signature decides after the read-back below).
    int provisional = -1;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        const Sig lo = signature(p, 0);
        for (auto it = g_tune.lower_bound(lo); it != g_tune.end() && it->first.same_size(lo); ++it)
            if (spmv_config(dtype, it->second.cfg).kind != 3) {
                provisional = it->second.cfg;
                break;
            }
    }
    // one allocation for the launch state and the build's readback words;
    // the whole build (validation, longest row, first partition, carry
    // slots) is queued on s and read back with one synchronization
    static_assert(sizeof(LaunchState) % alignof(PlanScratch) == 0, "scratch alignment");
    int st = dev_alloc(&p->state, sizeof(LaunchState) + sizeof(PlanScratch), s);
    if (st != MERBIT_OK) {
        delete p;
        return st;
    }
    p->scratch = reinterpret_cast<PlanScratch*>(p->state + 1);
    struct {
        LaunchState ls;
        PlanScratch sc;
    } init = {};
    static_assert(sizeof(init) == sizeof(LaunchState) + sizeof(PlanScratch), "state layout");
    init.ls.epoch = 1u;
    init.sc = PlanScratch{0, {INT_MAX, INT_MAX}, 0, 0, 0};
    cudaError_t e = cudaMemcpyAsync(p->state, &init, sizeof(init), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
        merbit_plan_destroy(p);
        return cuda_fail(e, "plan_create: init state");
    }
    const bool validate = !(flags & MERBIT_PLAN_SKIP_VALIDATE);
    st = validate_launch(d_row_ptr, d_col_idx, nrow, ncol, nnz, p->scratch, validate, s);
    // first candidate: the provisional cached configuration, else the
    // table's first entry the plan's alignment allows
    int first = -1;
    if (provisional >= 0 && spmv_config_allowed(spmv_config(dtype, provisional), p->vec))
        first = provisional;
    for (int i = 0, n = spmv_num_configs(dtype); first < 0 && i < n; ++i)
        if (spmv_config_allowed(spmv_config(dtype, i), p->vec)) first = i;
    Partition* part = nullptr;
    if (st == MERBIT_OK && first >= 0 && spmv_config(dtype, first).kind != 3)
        st = plan_partition_start(p, spmv_tile_items(spmv_config(dtype, first)), &part, s);
    PlanScratch h = {};
    if (st == MERBIT_OK) {
        e = cudaMemcpyAsync(&h, p->scratch, sizeof(h), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "plan_create: readback");
    }
    if (st == MERBIT_OK && validate) st = validate_status(h);
    if (st == MERBIT_OK) {
        p->max_row_len = h.max_row_len;
        if (part) part->max_rows = h.max_rows;
        // the exact signature, longest row included
        int tuned = -1;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto it = g_tune.find(signature(p, p->max_row_len));
            if (it != g_tune.end() && cached_choice_fits(dtype, it->second, p->max_row_len))
                tuned = it->second.cfg;
        }
        bool ok = false;
        if (tuned >= 0) {
            st = plan_config_ok(p, tuned, &ok, s);  // reuses the partition built above
            if (st == MERBIT_OK && ok) p->cfg = tuned;
        } else {
            // no cached choice for this signature: the provisional one came
            // from another longest-row bucket, so it is not kept
            const bool from_cache = first == provisional && provisional >= 0;
            ok = !from_cache && first >= 0 &&
                 (!part || h.max_rows <= spmv_config_row_cap(spmv_config(dtype, first)));
            if (ok) p->cfg = first;
        }
        if (st == MERBIT_OK && !ok) st = plan_pick_default(p, s);  // reuses built partitions
    }
    if (st != MERBIT_OK) {
        merbit_plan_destroy(p);
        return st;
    }
    *plan = p;
    return MERBIT_OK;
}

int merbit_plan_destroy(merbit_plan plan) {
    if (!plan) return MERBIT_OK;
    // the plan's launches may still run on any stream: wait for the device,
    // as cudaFree does, then hand the blocks back to the pool
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != plan->device) cudaSetDevice(plan->device);
    cudaDeviceSynchronize();
    for (auto& q : plan->parts) dev_free(q.coords, nullptr);
    for (auto& kv : plan->spmm_slots) {
        dev_free(kv.second.words, nullptr);
        dev_free(kv.second.state, nullptr);
    }
    dev_free(plan->carry, nullptr);
    dev_free(plan->state, nullptr);
    dev_free(plan->row_of, nullptr);
    dev_free(plan->partials, nullptr);
    for (void* q : plan->owned) dev_free(q, nullptr);
    if (cur != plan->device) cudaSetDevice(cur);
    delete plan;
    return MERBIT_OK;
}

int merbit_plan_get_info(merbit_plan plan, merbit_plan_info* info) {
    if (!plan || !info) return fail(MERBIT_ERR_INVALID, "plan_get_info: null pointer");
    const SpmvConfig c = spmv_config(plan->dtype, plan->cfg);
    info->nrow = plan->nrow;
    info->ncol = plan->ncol;
    info->nnz = plan->nnz;
    info->dtype = plan->dtype;
    info->block = c.block;
    info->items_per_thread = c.ipt;
    info->tile_items = spmv_tile_items(c);
    info->num_tiles = 0;
    int64_t meta = sizeof(LaunchState) + (int64_t)plan->slots * 4 * (int64_t)sizeof(unsigned long long);
    for (auto& q : plan->parts) {
        if (q.tile_items == info->tile_items) info->num_tiles = q.num_tiles;
        meta += (int64_t)(q.num_tiles + 1) * (int64_t)sizeof(int2);
    }
    info->vectorized = plan->vec ? 1 : 0;
    info->kind = c.kind;
    info->l1_carveout = c.carveout;
    info->gather_l2_only = c.cg;
    info->metadata_bytes = meta;
    info->max_row_len = plan->max_row_len;
    info->algorithmic_bytes = 4.0 * (plan->nrow + 1.0) +
                              (double)plan->nnz * (4.0 + (double)dtype_size(plan->dtype)) +
                              (double)xy_size(plan->dtype) * ((double)plan->ncol + plan->nrow);
    return MERBIT_OK;
}

int merbit_plan_set_values(merbit_plan plan, const void* d_vals) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "plan_set_values: plan is null");
    if (plan->nnz > 0 && !d_vals) return fail(MERBIT_ERR_INVALID, "plan_set_values: vals is null");
    plan->vals = d_vals;
    plan->vec = aligned16(plan->col) && aligned16(d_vals) && aligned16(plan->row_ptr);
    bool ok = false;
    int st = plan_config_ok(plan, plan->cfg, &ok, nullptr);
    if (st == MERBIT_OK && !ok) st = plan_pick_default(plan, nullptr);
    return st;
}

int merbit_spmv(merbit_plan plan, double alpha, const void* d_x, double beta, void* d_y,
                void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "spmv: plan is null");
    if (plan->nrow == 0) return MERBIT_OK;
    if (!d_y || (plan->ncol > 0 && !d_x)) return fail(MERBIT_ERR_INVALID, "spmv: x/y is null");
    return run_spmv(plan, plan->cfg, alpha, d_x, beta, d_y, (cudaStream_t)stream);
}

int merbit_pagerank_step(merbit_plan plan, double damp, const void* d_x, const void* d_teleport,
                         void* d_y, double* d_residual, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "pagerank_step: plan is null");
    if (plan->nrow != plan->ncol) return fail(MERBIT_ERR_INVALID, "pagerank_step: plan is not square");
    if (plan->nrow == 0) {
        if (d_residual) MERBIT_CUDA(cudaMemsetAsync(d_residual, 0, sizeof(double), (cudaStream_t)stream));
        return MERBIT_OK;
    }
    if (!d_x || !d_y || !d_teleport) return fail(MERBIT_ERR_INVALID, "pagerank_step: null vector");
    if (d_x == d_y) return fail(MERBIT_ERR_INVALID, "pagerank_step: x and y must differ");
    if (!(damp >= 0.0 && damp <= 1.0)) return fail(MERBIT_ERR_INVALID, "pagerank_step: damp outside [0, 1]");
    // on the plan's device for this call; the caller's current device is restored
    int cur = 0;
    MERBIT_CUDA(cudaGetDevice(&cur));
    if (cur != plan->device) MERBIT_CUDA(cudaSetDevice(plan->device));
    const int st = run_spmv(plan, plan->cfg, damp, d_x, 1.0 - damp, d_y, (cudaStream_t)stream,
                            d_teleport, d_residual);
    if (cur != plan->device) cudaSetDevice(cur);
    return st;
}

int merbit_plan_tune(merbit_plan plan, const void* d_x, void* d_y, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "plan_tune: plan is null");
    if (plan->nrow == 0) return MERBIT_OK;
    if (!d_y || (plan->ncol > 0 && !d_x)) return fail(MERBIT_ERR_INVALID, "plan_tune: x/y is null");
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    MERBIT_CUDA(cudaEventCreate(&e0));
    MERBIT_CUDA(cudaEventCreate(&e1));
    const int n = spmv_num_configs(plan->dtype);
    int best = plan->cfg;
    int st = MERBIT_OK;
    // ms of `reps` back-to-back launches of configuration c
    auto time_cfg = [&](int c, int reps, float* ms) -> int {
        int rc = MERBIT_OK;
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps && rc == MERBIT_OK; ++r) rc = run_spmv(plan, c, 1.0, d_x, 0.0, d_y, s);
        cudaEventRecord(e1, s);
        cudaError_t ce = cudaEventSynchronize(e1);
        if (ce != cudaSuccess) return cuda_fail(ce, "plan_tune");
        if (rc != MERBIT_OK) return rc;
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= (float)reps;
        return MERBIT_OK;
    };
    // 1. every usable configuration, 5 launches after 2 warm-up launches
    std::vector<std::pair<float, int>> timed;
    for (int c = 0; c < n && st == MERBIT_OK; ++c) {
        bool ok = false;
        st = plan_config_ok(plan, c, &ok, s);
        if (st != MERBIT_OK) break;
        if (!ok) continue;
        for (int w = 0; w < 2 && st == MERBIT_OK; ++w) st = run_spmv(plan, c, 1.0, d_x, 0.0, d_y, s);
        float ms = 0.f;
        if (st == MERBIT_OK) st = time_cfg(c, 5, &ms);
        if (st == MERBIT_OK) timed.push_back({ms, c});
    }
    // 2. the three fastest again, best of three rounds of 10 launches each
    //    (a single short round cannot separate entries within a few percent)
    if (st == MERBIT_OK && !timed.empty()) {
        std::stable_sort(timed.begin(), timed.end());
        const size_t top = std::min<size_t>(3, timed.size());
        float best_ms = 1e30f;
        best = timed[0].second;
        for (int round = 0; round < 3 && st == MERBIT_OK; ++round)
            for (size_t i = 0; i < top && st == MERBIT_OK; ++i) {
                float ms = 0.f;
                st = time_cfg(timed[i].second, 10, &ms);
                if (st == MERBIT_OK && ms < best_ms) {
                    best_ms = ms;
                    best = timed[i].second;
                }
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != MERBIT_OK) return st;
    plan->cfg = best;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[signature(plan, plan->max_row_len)] = Tuned{best, plan->max_row_len};
    return MERBIT_OK;
}

int merbit_num_configs(merbit_dtype dtype) {
    if (dtype != MERBIT_F64 && dtype != MERBIT_F32 && dtype != MERBIT_BF16) return 0;
    return spmv_num_configs(dtype);
}

int merbit_config_desc(merbit_dtype dtype, int32_t idx, int32_t* kind, int32_t* block,
                       int32_t* items_per_thread) {
    if (idx < 0 || idx >= merbit_num_configs(dtype) || !kind || !block || !items_per_thread)
        return fail(MERBIT_ERR_INVALID, "config_desc: bad index");
    const SpmvConfig c = spmv_config(dtype, idx);
    *kind = c.kind;
    *block = c.block;
    *items_per_thread = c.ipt;
    return MERBIT_OK;
}

int merbit_plan_set_config(merbit_plan plan, int32_t idx, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "plan_set_config: plan is null");
    if (idx < 0 || idx >= spmv_num_configs(plan->dtype))
        return fail(MERBIT_ERR_INVALID, "plan_set_config: bad index");
    bool ok = false;
    int st = plan_config_ok(plan, idx, &ok, (cudaStream_t)stream);
    if (st != MERBIT_OK) return st;
    if (!ok)
        return fail(MERBIT_ERR_INVALID,
                    "plan_set_config: configuration cannot run this plan (needs 16-byte aligned "
                    "arrays, or the matrix ends too many rows in one tile)");
    plan->cfg = idx;
    return MERBIT_OK;
}

int merbit_plan_config_usable(merbit_plan plan, int32_t idx, int32_t* usable, void* stream) {
    if (!plan || !usable) return fail(MERBIT_ERR_INVALID, "plan_config_usable: null pointer");
    if (idx < 0 || idx >= spmv_num_configs(plan->dtype))
        return fail(MERBIT_ERR_INVALID, "plan_config_usable: bad index");
    bool ok = false;
    int st = plan_config_ok(plan, idx, &ok, (cudaStream_t)stream);
    *usable = ok ? 1 : 0;
    return st;
}

int merbit_plan_check(merbit_plan plan, void* stream) {
    if (!plan) return fail(MERBIT_ERR_INVALID, "plan_check: plan is null");
    cudaStream_t s = (cudaStream_t)stream;
    int err = 0;
    MERBIT_CUDA(cudaMemcpyAsync(&err, &plan->state->error, sizeof(int), cudaMemcpyDeviceToHost, s));
    MERBIT_CUDA(cudaStreamSynchronize(s));
    if (err != 0) {
        const int zero = 0;
        MERBIT_CUDA(cudaMemcpyAsync(&plan->state->error, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
        MERBIT_CUDA(cudaStreamSynchronize(s));
        return fail(err, "a device-side carry wait ran out");
    }
    return MERBIT_OK;
}

}  // extern "C"
