// batch.cpp -- many helical scans of uneven size reconstructed together.
//
// A batch holds one filter plan and one backprojection plan per scan, the PI tables of all
// scans, and a device array describing every scan to the persistent backprojector
// (k_bkproj2_batch): per run, the scans' filters and PI solves are enqueued one after the
// other, then ONE persistent launch backprojects the tiles of all scans, CTAs pulling tiles
// from a shared counter (scans sorted largest first, so the small ones fill the tail). With
// use_graph, the first run is executed eagerly (it sizes every work buffer) and the second is
// captured into a CUDA graph that later runs replay; the graph is re-captured when the buffer
// pointers change. Scans on the fifth form (10..12) get their cell records written right
// before the persistent launch (the records of all of a group's scans are held at once).
#include "internal.h"

#include <algorithm>
#include <cstring>
#include <memory>
#include <numeric>
#include <vector>

namespace ctr {
Status launch_bkproj_batch(int variant, cudaStream_t s, const BatchScanDev* d_scans, int n,
                           long long total, unsigned long long* d_counter, int cells_cap,
                           int raw_cap, int* err);
long long bkproj_batch_tiles(const BPParams& kp, int variant);
Status launch_pi_stats(ctrecon_ctx* ctx, cudaStream_t s, BPPlan& plan, PiRecord* d_pitab,
                       unsigned long long* d_updates, unsigned long long* d_iters);
void set_noctx_error(const std::string& m);
}  // namespace ctr

using namespace ctr;

// Scans that share a backprojector form: one persistent launch over their tiles.
struct BatchGroup {
    int variant = 0;
    int nscans = 0;
    long long tiles = 0;
    int cells = 0, raw = 0;  // fourth-form staging capacities (largest over the group); the
                             // fifth form's box capacity in `cells`
    DevBuf table, counter;
    // fifth form: every scan's cell records and box-map table
    DevBuf rec, maps;
    struct RecJob { const float* fproj; void* rec; int P, YL, ZL; };
    std::vector<RecJob> jobs;
};

struct ctrecon_batch {
    ctrecon_ctx* ctx = nullptr;
    int n = 0;
    std::vector<int> svar;            // backprojector form of each scan
    std::vector<ctrecon_filter_params> fp;
    std::vector<std::unique_ptr<FilterPlan>> fplans;
    std::vector<std::unique_ptr<BPPlan>> bplans;
    std::vector<int> order;           // scans by decreasing backprojection work
    std::vector<size_t> pit_off;      // PiRecord offset of each scan in `pitab`
    DevBuf pitab, updates;
    // groups of scans by form (rebuilt by upload_scans; the buffers are reused)
    std::vector<std::unique_ptr<BatchGroup>> groups;
    int ngroups = 0;
    // what the graph was captured with: the buffer pointers, the context options, the
    // learned-initialiser version and the work-buffer allocation epoch
    std::vector<unsigned long long> key;
    int runs_with_key = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~ctrecon_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

static ctrecon_status bfinish(ctrecon_ctx* ctx, const Status& s) {
    if (!s.ok()) {
        if (ctx) ctx->last_error = s.msg;
        else set_noctx_error(s.msg);
    }
    return s.code;
}

// one persistent backprojection launch per group of scans sharing a form (the scan tables
// must be uploaded)
static Status batch_backproject(ctrecon_batch* b, cudaStream_t s) {
    for (int g = 0; g < b->ngroups; ++g) {
        BatchGroup& G = *b->groups[g];
        for (const auto& j : G.jobs)
            CTR_TRY(launch_cell_records(s, j.fproj, j.rec, 0, j.P, j.YL, j.ZL));
        CTR_TRY(launch_bkproj_batch(G.variant, s, G.table.as<BatchScanDev>(), G.nscans, G.tiles,
                                    G.counter.as<unsigned long long>(), G.cells, G.raw,
                                    b->ctx->ws_flag.as<int>()));
    }
    return Status::Ok();
}

static Status enqueue(ctrecon_batch* b, cudaStream_t s, const float* const* d_proj,
                      float* const* d_fproj, float* const* d_image) {
    ctrecon_ctx* ctx = b->ctx;
    CTR_TRY(reset_device_flag(ctx, s));
    for (int k = 0; k < b->n; ++k) {
        const int i = b->order[k];
        const int P = b->fp[i].proj_number;
        CTR_TRY(launch_filter(ctx, s, *b->fplans[i], d_proj[i], 0, P, d_fproj[i], 0, 0, P));
    }
    for (int k = 0; k < b->n; ++k) {
        const int i = b->order[k];
        CTR_TRY(launch_pi(ctx, s, *b->bplans[i], b->pitab.as<PiRecord>() + b->pit_off[i], nullptr));
    }
    return batch_backproject(b, s);
}

// Groups the scans by form (largest work first within a group) and uploads each group's scan
// table; the group buffers are reused, so a stable configuration allocates nothing.
static Status upload_scans(ctrecon_batch* b, cudaStream_t s, float* const* d_fproj,
                           float* const* d_image) {
    // The fifth form holds the cell records of all its scans at once: when they would take
    // more than half of the free device memory (beside what the batch already holds), its
    // largest scans move to the fourth form (variant 9) until they fit.
    {
        size_t held = 0;
        for (const auto& G : b->groups) held += G->rec.bytes;
        auto rec_of = [&](int i) {
            const BPParams& kp = b->bplans[i]->kp;
            return (size_t)kp.P * (kp.ZL - 1) * (kp.YL - 1) * 16;
        };
        std::vector<int> five;
        size_t need = 0;
        for (int i = 0; i < b->n; ++i)
            if (b->svar[i] >= 10) { five.push_back(i); need += rec_of(i); }
        // the driver is asked for free memory only when the batch would need more than it holds
        // (a query per run can stall the host while other processes hold the driver)
        size_t budget = need;
        if (need > held) {
            size_t free_b = 0, total_b = 0;
            CTR_CUDA(cudaMemGetInfo(&free_b, &total_b));
            budget = (free_b + held) / 2;
        }
        std::sort(five.begin(), five.end(), [&](int x, int y) { return rec_of(x) > rec_of(y); });
        for (size_t k = 0; k < five.size() && need > budget; ++k) {
            need -= rec_of(five[k]);
            b->svar[five[k]] = 9;
        }
    }
    std::vector<int> forms;
    for (int k = 0; k < b->n; ++k) {
        const int v = b->svar[b->order[k]];
        if (std::find(forms.begin(), forms.end(), v) == forms.end()) forms.push_back(v);
    }
    while (b->groups.size() < forms.size()) b->groups.emplace_back(new BatchGroup());
    b->ngroups = (int)forms.size();
    for (int g = 0; g < b->ngroups; ++g) {
        BatchGroup& G = *b->groups[g];
        G.variant = forms[g];
        std::vector<BatchScanDev> h;
        long long first = 0;
        int cells = 0, raw = 0;
        const bool rec = G.variant >= 10;
        size_t rec_bytes = 0;
        if (rec)
            for (int k = 0; k < b->n; ++k) {
                const int i = b->order[k];
                if (b->svar[i] != G.variant) continue;
                const BPParams& kp = b->bplans[i]->kp;
                rec_bytes += (size_t)kp.P * (kp.ZL - 1) * (kp.YL - 1) * 16;
            }
        std::vector<unsigned char> hmaps;
        size_t rec_off = 0;
        G.jobs.clear();
        if (rec) {
            CTR_TRY(G.rec.ensure(rec_bytes, "batch cell records"));
            int ns = 0;
            for (int k = 0; k < b->n; ++k) ns += b->svar[b->order[k]] == G.variant;
            CTR_TRY(G.maps.ensure((size_t)ns * kBoxMaps * 128, "batch box maps"));
            hmaps.assign((size_t)ns * kBoxMaps * 128, 0);
        }
        for (int k = 0; k < b->n; ++k) {
            const int i = b->order[k];
            if (b->svar[i] != G.variant) continue;
            BPPlan& bp = *b->bplans[i];
            BatchScanDev d;
            d.kp = bp.kp;
            d.fproj = d_fproj[i];
            d.pit = b->pitab.as<PiRecord>() + b->pit_off[i];
            d.views = bp.views.as<float4>();
            d.xyz = bp.xyz.as<float>();
            d.image = d_image[i];
            d.first_tile = first;
            d.tmaps = nullptr;
            d.rec_p0 = 0;
            first += bkproj_batch_tiles(bp.kp, G.variant);
            bp4_caps(bp);
            if (rec) {
                const BPParams& kp = bp.kp;
                unsigned char* r = G.rec.as<unsigned char>() + rec_off;
                rec_off += (size_t)kp.P * (kp.ZL - 1) * (kp.YL - 1) * 16;
                const size_t mi = h.size() * kBoxMaps * 128;
                CTR_TRY(encode_box_maps(hmaps.data() + mi, r, kp.YL - 1, kp.ZL - 1, kp.P));
                d.tmaps = G.maps.as<unsigned char>() + mi;
                G.jobs.push_back({d_fproj[i], r, kp.P, kp.YL, kp.ZL});
                cells = std::max(cells, bp.caps_box);
            } else {
                cells = std::max(cells, bp.caps_cells);
                raw = std::max(raw, bp.caps_raw);
            }
            h.push_back(d);
        }
        G.nscans = (int)h.size();
        G.tiles = first;
        G.cells = cells;
        G.raw = raw;
        CTR_TRY(G.table.ensure(h.size() * sizeof(BatchScanDev), "batch scan table"));
        CTR_TRY(G.counter.ensure(64, "batch work counter"));
        CTR_CUDA(cudaMemcpyAsync(G.table.ptr, h.data(), h.size() * sizeof(BatchScanDev),
                                 cudaMemcpyHostToDevice, s));
        if (rec)
            CTR_CUDA(cudaMemcpyAsync(G.maps.ptr, hmaps.data(), hmaps.size(),
                                     cudaMemcpyHostToDevice, s));
        CTR_CUDA(cudaStreamSynchronize(s));  // `h` and `hmaps` are pageable and local
    }
    return Status::Ok();
}

extern "C" {

ctrecon_status ctrecon_batch_create(ctrecon_ctx* ctx, int n_scans,
                                    const ctrecon_filter_params* fp, const ctrecon_bp_geom* g,
                                    ctrecon_batch** out) {
    if (!ctx || !fp || !g || !out || n_scans < 1) return CTRECON_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        cudaSetDevice(ctx->device);
        auto b = std::make_unique<ctrecon_batch>();
        b->ctx = ctx;
        b->n = n_scans;
        b->svar.assign(n_scans, (ctx->opt_bp_variant >= 0 && ctx->opt_bp_variant <= kMaxBPVariant)
                                    ? ctx->opt_bp_variant
                                    : kDefaultBatchVariant);
        b->fp.assign(fp, fp + n_scans);
        size_t nvox = 0;
        std::vector<double> work(n_scans);
        for (int i = 0; i < n_scans; ++i) {
            b->fplans.emplace_back(new FilterPlan());
            b->bplans.emplace_back(new BPPlan());
            Status s = build_filter_plan(fp[i], *b->fplans[i]);
            BPGeom bg;
            std::memset(&bg, 0, sizeof bg);
            if (s.ok()) s = parse_bp_geom(g[i], bg);
            if (s.ok() && (bg.YL != fp[i].yl || bg.ZL != fp[i].zl || bg.ProjNum != fp[i].proj_number))
                s = make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                "scan " + std::to_string(i) + ": filter and geometry disagree");
            if (s.ok()) s = build_bp_plan(bg, *b->bplans[i]);
            if (!s.ok()) return bfinish(ctx, s);
            b->pit_off.push_back(nvox);
            nvox += (size_t)bg.NX * bg.NY * bg.NZ;
            work[i] = (double)bg.NX * bg.NY * bg.NZ * bg.ProjScale;
        }
        b->order.resize(n_scans);
        std::iota(b->order.begin(), b->order.end(), 0);
        std::stable_sort(b->order.begin(), b->order.end(),
                         [&](int a, int c) { return work[a] > work[c]; });
        Status s = b->pitab.ensure(nvox * sizeof(PiRecord), "batch PI tables");
        if (s.ok()) s = b->updates.ensure(sizeof(unsigned long long) * n_scans, "batch counts");
        if (!s.ok()) return bfinish(ctx, s);
        *out = b.release();
        return CTRECON_OK;
    } catch (const std::exception& e) {
        return bfinish(ctx, make_status(CTRECON_ERR_INTERNAL, e.what()));
    }
}

void ctrecon_batch_destroy(ctrecon_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    delete b;
}

ctrecon_status ctrecon_batch_set_variant(ctrecon_batch* b, int variant) {
    if (!b || variant < 0 || variant > kMaxBPVariant) return CTRECON_ERR_INVALID_ARGUMENT;
    for (int& v : b->svar) v = variant;
    b->key.clear();  // tile counts change: rebuild the scan tables and the graph
    return CTRECON_OK;
}

ctrecon_status ctrecon_batch_set_variants(ctrecon_batch* b, const int* variants, int n) {
    if (!b || !variants || n != b->n) return CTRECON_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n; ++i)
        if (variants[i] < 0 || variants[i] > kMaxBPVariant) return CTRECON_ERR_INVALID_ARGUMENT;
    b->svar.assign(variants, variants + n);
    b->key.clear();
    return CTRECON_OK;
}

ctrecon_status ctrecon_batch_get_variants(const ctrecon_batch* b, int* variants, int n) {
    if (!b || !variants || n < b->n) return CTRECON_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < b->n; ++i) variants[i] = b->svar[i];
    return CTRECON_OK;
}

ctrecon_status ctrecon_batch_run_dev(ctrecon_batch* b, void* stream, const float* const* d_proj,
                                     float* const* d_fproj, float* const* d_image,
                                     int use_graph) {
    if (!b || !d_proj || !d_fproj || !d_image) return CTRECON_ERR_INVALID_ARGUMENT;
    ctrecon_ctx* ctx = b->ctx;
    try {
        cudaSetDevice(ctx->device);
        cudaStream_t s = (cudaStream_t)stream;
        if (use_graph && !s)
            return bfinish(ctx, make_status(CTRECON_ERR_INVALID_ARGUMENT,
                                            "graph replay needs a created stream, not stream 0"));
        std::vector<unsigned long long> key;
        for (int i = 0; i < b->n; ++i) {
            key.push_back((uintptr_t)d_proj[i]);
            key.push_back((uintptr_t)d_fproj[i]);
            key.push_back((uintptr_t)d_image[i]);
        }
        key.push_back((unsigned long long)ctx->opt_hilbert);
        key.push_back((unsigned long long)ctx->opt_pi);
        key.push_back((unsigned long long)ctx->opt_filter_chunk);
        key.push_back((unsigned long long)ctx->pinet.version);
        key.push_back(devbuf_epoch());
        if (key != b->key) {
            Status st = upload_scans(b, s, d_fproj, d_image);
            if (!st.ok()) return bfinish(ctx, st);
            b->key = key;
            b->runs_with_key = 0;
            if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
            if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
        }
        Status st;
        if (!use_graph || b->runs_with_key == 0) {
            st = enqueue(b, s, d_proj, d_fproj, d_image);
        } else {
            if (!b->exec) {
                cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) return bfinish(ctx, cuda_status(e, "cudaStreamBeginCapture"));
                st = enqueue(b, s, d_proj, d_fproj, d_image);
                cudaGraph_t g = nullptr;
                e = cudaStreamEndCapture(s, &g);
                if (st.ok() && e != cudaSuccess) st = cuda_status(e, "cudaStreamEndCapture");
                if (st.ok()) {
                    e = cudaGraphInstantiate(&b->exec, g, 0);
                    if (e != cudaSuccess) st = cuda_status(e, "cudaGraphInstantiate");
                }
                b->graph = g;
                if (!st.ok()) return bfinish(ctx, st);
            }
            cudaError_t e = cudaGraphLaunch(b->exec, s);
            if (e != cudaSuccess) st = cuda_status(e, "cudaGraphLaunch");
        }
        if (st.ok()) b->runs_with_key++;
        return bfinish(ctx, st);
    } catch (const std::exception& e) {
        return bfinish(ctx, make_status(CTRECON_ERR_INTERNAL, e.what()));
    }
}

ctrecon_status ctrecon_batch_tune(ctrecon_batch* b, void* stream, const float* const* d_proj,
                                  float* const* d_fproj, float* const* d_image,
                                  ctrecon_tune_result* out) {
    if (!b || !d_proj || !d_fproj || !d_image || !out) return CTRECON_ERR_INVALID_ARGUMENT;
    ctrecon_ctx* ctx = b->ctx;
    try {
        cudaSetDevice(ctx->device);
        cudaStream_t s = (cudaStream_t)stream;
        // one eager run: filters, PI solves and a backprojection with the current forms
        ctrecon_status rc = ctrecon_batch_run_dev(b, stream, d_proj, d_fproj, d_image, 0);
        if (rc != CTRECON_OK) return rc;
        // each scan's form: every candidate timed on that scan alone (single-scan launches)
        std::memset(out, 0, sizeof *out);
        const int saved_opt = ctx->opt_bp_variant;
        Status st;
        std::vector<int> best(b->n, kDefaultBatchVariant);
        double best_sum = 0;
        std::vector<double> cand_sum;
        for (int i = 0; st.ok() && i < b->n; ++i) {
            ctrecon_tune_result r;
            st = tune_candidates(&r, s, nullptr, [&](int v) {
                ctx->opt_bp_variant = v;
                return launch_bkproj_f32(ctx, s, *b->bplans[i],
                                         d_fproj[i], b->pitab.as<PiRecord>() + b->pit_off[i],
                                         d_image[i]);
            });
            if (!st.ok()) break;
            best[i] = r.best_variant;
            best_sum += r.best_ms;
            if (cand_sum.empty()) {
                out->n = r.n;
                cand_sum.assign(r.n, 0.0);
                for (int c = 0; c < r.n; ++c) out->variants[c] = r.variants[c];
            }
            for (int c = 0; c < r.n; ++c)
                cand_sum[c] = (cand_sum[c] < 0 || r.ms[c] < 0) ? -1.0 : cand_sum[c] + r.ms[c];
        }
        ctx->opt_bp_variant = saved_opt;
        if (st.ok()) {
            b->svar = best;
            for (int c = 0; c < out->n; ++c) out->ms[c] = (float)cand_sum[c];
            out->best_ms = (float)best_sum;  // sum of the scans' best single-scan times
            // the form that covers most scans
            int most = best[0], cnt = 0;
            for (int v : best) {
                const int k = (int)std::count(best.begin(), best.end(), v);
                if (k > cnt) { cnt = k; most = v; }
            }
            out->best_variant = most;
            // leave the winners' backprojections in the images
            st = upload_scans(b, s, d_fproj, d_image);
            if (st.ok()) st = batch_backproject(b, s);
            if (st.ok()) {
                cudaError_t e = cudaStreamSynchronize(s);
                if (e != cudaSuccess) st = cuda_status(e, "cudaStreamSynchronize");
            }
        }
        b->key.clear();  // the next run re-uploads the scan table and re-captures its graph
        if (st.ok()) {
            int flag = 0;
            cudaError_t e = cudaMemcpy(&flag, ctx->ws_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) st = cuda_status(e, "device error word");
            else if (flag) st = make_status(CTRECON_ERR_TIMEOUT, "a device-side wait gave up");
        }
        return bfinish(ctx, st);
    } catch (const std::exception& e) {
        return bfinish(ctx, make_status(CTRECON_ERR_INTERNAL, e.what()));
    }
}

ctrecon_status ctrecon_batch_updates(ctrecon_batch* b, unsigned long long* host_updates) {
    if (!b || !host_updates) return CTRECON_ERR_INVALID_ARGUMENT;
    ctrecon_ctx* ctx = b->ctx;
    try {
        cudaSetDevice(ctx->device);
        cudaStream_t s = ctx->host_stream;
        const int saved = ctx->opt_pi;
        ctx->opt_pi = CTRECON_PI_BISECT;  // the loop count of the reference's own solve
        Status st = reset_device_flag(ctx, s);
        cudaError_t e0 = st.ok() ? cudaMemsetAsync(b->updates.ptr, 0,
                                                   sizeof(unsigned long long) * b->n, s)
                                 : cudaSuccess;
        if (e0 != cudaSuccess) st = cuda_status(e0, "batch counts");
        for (int i = 0; st.ok() && i < b->n; ++i)
            st = launch_pi_stats(ctx, s, *b->bplans[i], b->pitab.as<PiRecord>() + b->pit_off[i],
                                 b->updates.as<unsigned long long>() + i, nullptr);
        ctx->opt_pi = saved;
        if (st.ok()) {
            cudaError_t e = cudaMemcpyAsync(host_updates, b->updates.ptr,
                                            sizeof(unsigned long long) * b->n,
                                            cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) st = cuda_status(e, "batch counts");
        }
        return bfinish(ctx, st);
    } catch (const std::exception& e) {
        return bfinish(ctx, make_status(CTRECON_ERR_INTERNAL, e.what()));
    }
}

}  // extern "C"
