// recon.cu -- end-to-end streaming FDK on one GPU: the single-GPU analogue of cuFDK's
// FilterThread -> BpThread handoff (cuFDK/mpiFDK.cpp:58-317).
//
//   host views --(copy stream, a ring of raw-view slots)--> raw views on the device
//   --(compute stream)--> fused cosine weight + ramp filter, written straight into the
//   backprojection's layout --> backprojection into the resident volume.
//
// Views move in chunks of up to 32; the ring holds batch / chunk + 2 chunks, so the copies of
// the next batch's views land while the current batch's backprojection runs (a slot is free
// again once its chunk is filtered, and the filters of a batch queue behind the previous
// batch's backprojection on the compute stream).  A full batch is held until the next batch
// starts, so at the end of a scan two batches wait, and the final flush runs them z band by z
// band: the volume's first bands are final early and their copy to the host overlaps the rest.
//
// The whole volume is one mirror-symmetric slab pair (DivVolume with one rank,
// cuFDK/mpiFDK.h:116-149): top = z in [0, nz/2), bottom = z in [nz/2, nz).  Host waits are
// bounded: fdk_recon_sync polls with a deadline and returns FDK_ERR_TIMEOUT instead of hanging.
#include <cuda_fp16.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

#include "common.h"
#include "internal.h"

using namespace fdk;

struct fdk_recon {
    fdk_geometry g{};
    int precision = FDK_BP_FP32;
    int batch = 32;
    int device = 0;
    int pad = 4;  // edge pad of the production IPP filter plugin (Filterlib/FilterLib.h:38,44)
    int layout = FDK_LAYOUT_MIRROR;
    int dtype = FDK_DTYPE_F32;
    fdk_bp *bp = nullptr;
    FilterTables tables;
    float *d_cos = nullptr;
    fdk_toeplitz *tpz = nullptr;     // tensor-core filter (MIXED), else the FFT filter
    int chunk = 32;                  // views per raw slot
    std::vector<float *> d_raw;      // the ring of raw-view slots
    void *d_filt[2] = {nullptr, nullptr};  // filtered-view batches: the one filling and the held one
    float *d_scale = nullptr;        // accumulator scale of FP16 views (device scalar)
    unsigned int *d_overflow = nullptr;
    float out_scale = 1.0f;
    std::vector<float> mats;         // 12 x n_proj, FP32 (from FP64)
    float *d_mats = nullptr;         // the same on the device
    cudaStream_t compute = nullptr, copy = nullptr;
    std::vector<cudaEvent_t> raw_ready, raw_free;
    cudaEvent_t done = nullptr;
    int slot = 0;
    // d_filt[cur] is filling: views bviews[cur] (pending of them, in arrival order).  held:
    // d_filt[cur ^ 1] holds a full batch that is backprojected when the next batch starts, or
    // together with the filling one at a flush (band-interleaved, see flush_all).  FP32_EXACT
    // batches hold consecutive views (its kernel reads a contiguous run of matrices); the staged
    // precisions take views in any order and pair them into quarter-turn quadruples at launch.
    int cur = 0;
    int pending = 0;
    bool held = false;
    // first batch of a scan streamed from host memory (staged precisions, batches of 128 or more):
    // 0 = not decided (no view since creation or reset), 1 = filling a quarter-size first batch,
    // launched as soon as it is full, 2 = regular batches
    int ramp = 0;
    std::vector<int> bviews[2];
    int sym_rot = 0;  // quarter-turn kernel's column map (0: not available for this scan)
    double filter_ms = 0;
    long long views = 0;
    long long filter_launches = 0;   // kernel launches of the filter since creation or reset
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ftimers;
    // pinned staging of fdk_recon_push_folder (allocated on first use): two chunks
    float *h_stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_free[2] = {nullptr, nullptr};
    cudaEvent_t sync_ev[2] = {nullptr, nullptr};  // scratch events of the bounded host waits
    unsigned int *h_word = nullptr;               // pinned host copy of the overflow flag
};

// internal hooks (bp.cu)
int fdk_bp_sym_setup_internal(fdk_bp *h, const float *mats, int n_proj, int *rot);
int fdk_bp_bp_lists_internal(fdk_bp *h, const void *views, int n_slots, const float *d_mats, const float *host_mats,
                             const int *s_slot, const int *s_view, int n_single, const int *q_slot,
                             const int *q_view, int n_quad, void *stream, int band);
int fdk_bp_set_acc_scale_internal(fdk_bp *h, const float *d_scale);
int fdk_bp_reserve_lerp_internal(fdk_bp *h, int n_slots);
int fdk_bp_choose_lerp_box_internal(fdk_bp *h, const float *mats, int n_proj);
long long fdk_bp_launches_internal(const fdk_bp *h);
int fdk_bp_bp_device_mats_internal(fdk_bp *h, const void *dev_proj, int32_t layout, const float *dev_mats,
                                   int32_t n_proj, const float *host_mats, void *stream, int32_t band);
int fdk_bp_band_count_internal(const fdk_bp *h);
int fdk_bp_check_internal(fdk_bp *h);

namespace {

int recon_release(fdk_recon *h) {
    if (!h) return FDK_OK;
    DeviceGuard dg(h->device);
    if (h->compute) cudaStreamSynchronize(h->compute);
    if (h->copy) cudaStreamSynchronize(h->copy);
    if (h->bp) fdk_bp_destroy(h->bp);
    if (h->tpz) fdk_toeplitz_destroy(h->tpz);
    h->tables.release();
    for (int i = 0; i < 2; i++) {
        if (h->h_stage[i]) cudaFreeHost(h->h_stage[i]);
        if (h->stage_free[i]) cudaEventDestroy(h->stage_free[i]);
    }
    for (float *p : h->d_raw)
        if (p) cudaFree(p);
    for (cudaEvent_t e : h->raw_ready)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->raw_free)
        if (e) cudaEventDestroy(e);
    for (auto &t : h->ftimers) {
        cudaEventDestroy(t.first);
        cudaEventDestroy(t.second);
    }
    if (h->d_cos) cudaFree(h->d_cos);
    if (h->d_mats) cudaFree(h->d_mats);
    for (void *p : h->d_filt)
        if (p) cudaFree(p);
    if (h->d_scale) cudaFree(h->d_scale);
    if (h->d_overflow) cudaFree(h->d_overflow);
    if (h->done) cudaEventDestroy(h->done);
    for (cudaEvent_t e : h->sync_ev)
        if (e) cudaEventDestroy(e);
    if (h->h_word) cudaFreeHost(h->h_word);
    if (h->compute) cudaStreamDestroy(h->compute);
    if (h->copy) cudaStreamDestroy(h->copy);
    delete h;
    return FDK_OK;
}

int collect_filter_timers(fdk_recon *h) {
    for (auto &t : h->ftimers) {
        FDK_TRY(wait_event(t.second, "filter"));
        float ms = 0;
        FDK_CUDA(cudaEventElapsedTime(&ms, t.first, t.second));
        h->filter_ms += ms;
        cudaEventDestroy(t.first);
        cudaEventDestroy(t.second);
    }
    h->ftimers.clear();
    return FDK_OK;
}

// Backproject the n filtered views of buffer b: every z band (band -1) or one, on the compute
// stream.  FP32_EXACT: one consecutive run.  Staged precisions: the views whose quarter-turn
// partners (v mod N/4 equal, one from each quarter of the scan) are in the same batch go to the
// quarter-turn kernel -- each such view as the base of one quadruple, its partners as the other
// three members -- the rest to the staged kernel by (slot, view).
int launch_batch(fdk_recon *h, int b, int n, int band) {
    const std::vector<int> &vw = h->bviews[b];
    if (h->precision == FDK_BP_FP32_EXACT) {
        const long long first = vw[0];
        return fdk_bp_bp_device_mats_internal(h->bp, h->d_filt[b], h->layout, h->d_mats + 12 * first, n,
                                              h->mats.data() + 12 * first, h->compute, band);
    }
    std::vector<int> s_slot, s_view, q_slot, q_view;
    if (h->sym_rot) {
        const int q = (int)(h->g.n_proj / 4);
        // (orbit, quarter, slot), grouped by orbit: complete quadruples take one slot per quarter
        std::vector<std::array<int, 3>> e(n);
        for (int i = 0; i < n; i++) e[i] = {vw[i] % q, vw[i] / q, i};
        std::sort(e.begin(), e.end());
        for (size_t i = 0; i < e.size();) {
            size_t j = i;
            while (j < e.size() && e[j][0] == e[i][0]) j++;
            std::vector<int> by_q[4];
            for (size_t k = i; k < j; k++) by_q[e[k][1]].push_back(e[k][2]);
            const size_t nq = std::min({by_q[0].size(), by_q[1].size(), by_q[2].size(), by_q[3].size()});
            for (size_t k = 0; k < nq; k++)
                // every member is the base view once: base p + mq with members p + (m + t)q, so
                // each view reaches every column (base columns c and their turns T^t(c))
                for (int m = 0; m < 4; m++) {
                    for (int t = 0; t < 4; t++) q_slot.push_back(by_q[(m + t) & 3][k]);
                    q_view.push_back(e[i][0] + m * q);
                }
            for (int t = 0; t < 4; t++)
                for (size_t k = nq; k < by_q[t].size(); k++) {
                    s_slot.push_back(by_q[t][k]);
                    s_view.push_back(vw[by_q[t][k]]);
                }
            i = j;
        }
    } else {
        for (int i = 0; i < n; i++) {
            s_slot.push_back(i);
            s_view.push_back(vw[i]);
        }
    }
    return fdk_bp_bp_lists_internal(h->bp, h->d_filt[b], h->batch, h->d_mats, h->mats.data(), s_slot.data(),
                                    s_view.data(), (int)s_slot.size(), q_slot.data(), q_view.data(),
                                    (int)q_view.size(), h->compute, band);
}

// The filling batch is full and more views arrive: backproject the held batch (its launch
// queues behind the filters already issued, and the next filters write its buffer after it),
// hold the full one, fill the other buffer.
int rotate_full(fdk_recon *h) {
    if (h->held) FDK_TRY(launch_batch(h, h->cur ^ 1, h->batch, -1));
    h->held = true;
    h->cur ^= 1;
    h->pending = 0;
    h->bviews[h->cur].clear();
    return FDK_OK;
}

// Backproject everything waiting.  With two batches waiting (the usual state after the last
// push of a scan) they run band by band, held then filling: z band 0 has all its views after two
// band launches instead of after the whole held batch, so a readback (fdk_bp_get_volume) starts
// early.  Each voxel still receives the held batch's views before the filling batch's.
int flush_all(fdk_recon *h) {
    if (h->held && h->pending > 0) {
        const int nb = fdk_bp_band_count_internal(h->bp);
        for (int b = 0; b < nb; b++) {
            FDK_TRY(launch_batch(h, h->cur ^ 1, h->batch, b));
            FDK_TRY(launch_batch(h, h->cur, h->pending, b));
        }
    } else if (h->held) {
        FDK_TRY(launch_batch(h, h->cur ^ 1, h->batch, -1));
    } else if (h->pending > 0) {
        FDK_TRY(launch_batch(h, h->cur, h->pending, -1));
    }
    h->held = false;
    h->pending = 0;
    if (h->ramp == 1) h->ramp = 2;
    h->bviews[0].clear();
    h->bviews[1].clear();
    return FDK_OK;
}

// Filter n raw views (device, consecutive in memory) with view indices ids[0..n) into the
// filling batch behind the views already there; a full batch is held until the next one starts
// (rotate_full).  FP32_EXACT: views join a batch only when they continue the waiting views (the
// next view expected); otherwise everything waiting is backprojected first.  Staged precisions:
// any views join.  host: the views came from host memory (a scan that starts so begins with a
// quarter-size batch).
int process_chunk(fdk_recon *h, const float *d_src, const int64_t *ids, int n, cudaEvent_t release, bool host) {
    const fdk_geometry &g = h->g;
    const long long frame = g.nu * g.nv;
    const long long dstride = h->layout == FDK_LAYOUT_MIRROR ? 2 * frame : frame;
    const size_t esz = h->dtype == FDK_DTYPE_F16 ? 2 : 4;
    const bool exact = h->precision == FDK_BP_FP32_EXACT;
    // A scan pushed from host memory starts with a quarter-size batch, backprojected as soon as
    // it is full, so the backprojection starts while the rest of the scan is still crossing PCIe
    // (a full first batch would be held until the next one starts).
    if (h->ramp == 0) h->ramp = (host && !exact && h->batch >= 128) ? 1 : 2;
    const int ramp_n = h->batch / 4;
    for (int done = 0; done < n;) {
        if (exact && (h->pending > 0 || h->held)) {
            const long long expected = h->pending > 0 ? (long long)h->bviews[h->cur].back() + 1
                                                      : (long long)h->bviews[h->cur ^ 1].back() + 1;
            if (ids[done] != expected) FDK_TRY(flush_all(h));
        }
        if (h->pending == h->batch) FDK_TRY(rotate_full(h));
        int m = std::min(n - done, h->batch - h->pending);
        if (h->ramp == 1) m = std::min(m, ramp_n - h->pending);
        if (exact) {  // one consecutive run at a time
            int r = 1;
            while (r < m && ids[done + r] == ids[done + r - 1] + 1) r++;
            m = r;
        }
        for (int i = 0; i < m; i++) h->bviews[h->cur].push_back((int)ids[done + i]);
        void *dst = static_cast<unsigned char *>(h->d_filt[h->cur]) + (size_t)h->pending * dstride * esz;
        std::pair<cudaEvent_t, cudaEvent_t> t;  // filter time only (the flush below is the BP's)
        FDK_CUDA(cudaEventCreate(&t.first));
        FDK_CUDA(cudaEventCreate(&t.second));
        FDK_CUDA(cudaEventRecord(t.first, h->compute));
        if (h->tpz)
            FDK_TRY(fdk_toeplitz_run_device(h->tpz, d_src + (long long)done * frame, dst, m, FDK_LAYOUT_MIRROR, 1.0f,
                                            h->compute));
        else
            FDK_TRY(filter_views(d_src + (long long)done * frame, (int)g.nu, frame, dst, (int)g.nv, dstride, h->d_cos,
                                 (int)g.nu, h->tables, (int)g.nu, (int)g.nv, h->pad, m, h->layout, h->dtype,
                                 h->compute, h->out_scale, h->d_overflow));
        FDK_CUDA(cudaEventRecord(t.second, h->compute));
        h->filter_launches += h->tpz ? 2 : 1;  // weighting pass + GEMM, or the fused FFT filter
        h->ftimers.push_back(t);
        h->pending += m;
        done += m;
        if (h->ramp == 1 && h->pending == ramp_n) {
            // the first batch goes now; the next fills the other buffer (its filters queue behind
            // this launch on the compute stream)
            FDK_TRY(launch_batch(h, h->cur, h->pending, -1));
            h->cur ^= 1;
            h->pending = 0;
            h->bviews[h->cur].clear();
            h->ramp = 2;
        }
    }
    if (h->ftimers.size() > 256) FDK_TRY(collect_filter_timers(h));
    // the raw views are consumed once filtered
    if (release) FDK_CUDA(cudaEventRecord(release, h->compute));
    h->views += n;
    return FDK_OK;
}

std::vector<int64_t> consecutive(int64_t first, int64_t n) {
    std::vector<int64_t> v(n);
    for (int64_t i = 0; i < n; i++) v[i] = first + i;
    return v;
}

// Host views through the copy ring: chunks of up to h->chunk views, each copied into a ring slot
// on the copy stream and filtered on the compute stream; returns once the last copy has landed.
int push_host(fdk_recon *h, const float *host_views, const int64_t *ids, int64_t n) {
    const long long frame = h->g.nu * h->g.nv;
    const int cap = h->chunk;
    cudaEvent_t last = nullptr;
    for (long long c = 0; c < n; c += cap) {
        const int m = (int)std::min<long long>(cap, n - c);
        const int k = h->slot;
        h->slot = (k + 1) % (int)h->d_raw.size();
        FDK_CUDA(cudaStreamWaitEvent(h->copy, h->raw_free[k], 0));
        FDK_CUDA(cudaMemcpyAsync(h->d_raw[k], host_views + c * frame, sizeof(float) * frame * m,
                                 cudaMemcpyHostToDevice, h->copy));
        FDK_CUDA(cudaEventRecord(h->raw_ready[k], h->copy));
        FDK_CUDA(cudaStreamWaitEvent(h->compute, h->raw_ready[k], 0));
        FDK_TRY(process_chunk(h, h->d_raw[k], ids + c, m, h->raw_free[k], true));
        last = h->raw_ready[k];
    }
    // the caller may reuse host_views once its last copy has landed
    if (last) FDK_TRY(wait_event(last, "view copy"));
    return FDK_OK;
}

int check_ids(const fdk_recon *h, const int64_t *ids, int64_t n) {
    for (int64_t i = 0; i < n; i++)
        FDK_CHECK_ARG(ids[i] >= 0 && ids[i] < h->g.n_proj, "view %lld outside 0..%lld", (long long)ids[i],
                      (long long)h->g.n_proj - 1);
    return FDK_OK;
}

}  // namespace

extern "C" {

int fdk_recon_create(fdk_recon **out, const fdk_geometry *g, int32_t precision, int32_t batch, int32_t device) {
    FDK_CHECK_ARG(g != nullptr, "NULL geometry");
    return fdk_recon_create_slab(out, g, 0, g->nz / 2, precision, batch, device);
}

int fdk_recon_stream(fdk_recon *h, void **stream) {
    FDK_CHECK_ARG(h && stream, "NULL argument");
    *stream = (void *)h->compute;
    return FDK_OK;
}

int fdk_recon_create_slab(fdk_recon **out, const fdk_geometry *g, int64_t top_z, int64_t depth, int32_t precision,
                          int32_t batch, int32_t device) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(out && g, "NULL argument");
    *out = nullptr;
    FDK_CHECK_ARG(precision >= FDK_BP_FP32_EXACT && precision <= FDK_BP_MIXED, "bad precision");
    FDK_CHECK_ARG(batch > 0 && batch <= 512, "batch must be 1..512");
    FDK_CHECK_ARG(g->nz % 2 == 0, "the slab-pair reconstructor needs an even nz");
    FDK_CHECK_ARG(depth > 0 && top_z >= 0 && top_z + depth <= g->nz / 2, "slab [%lld, %lld) outside the top half",
                  (long long)top_z, (long long)(top_z + depth));
    FDK_CHECK_ARG(g->nx <= 65535 * 16 && g->ny <= 65535 * 16, "volume too large");
    const int64_t W = fdk_filter_length(g->nu);
    FDK_CHECK_ARG(W <= 4096, "detector too wide: nextpow2(nu) = %lld > 4096", (long long)W);
    if (precision == FDK_BP_FP32_EXACT) FDK_CHECK_ARG(batch <= 32, "FP32_EXACT batches are <= 32 views");
    DeviceGuard dg(device);
    FDK_TRY(dg.status);
    fdk_recon *h = new fdk_recon();
    h->g = *g;
    h->precision = precision;
    h->batch = batch;
    h->device = device;
    h->layout = precision == FDK_BP_FP32_EXACT ? FDK_LAYOUT_TRANSPOSED : FDK_LAYOUT_MIRROR;
    h->dtype = precision == FDK_BP_MIXED ? FDK_DTYPE_F16 : FDK_DTYPE_F32;
    int s = FDK_OK;
    auto ck = [&](cudaError_t e, const char *what) {
        if (s == FDK_OK && e != cudaSuccess) s = cuda_status(e, what, __FILE__, __LINE__);
    };
    // the set-up copies below queue on the compute stream; the call waits for it at its end
    ck(cudaStreamCreateWithFlags(&h->compute, cudaStreamNonBlocking), "stream");
    if (s == FDK_OK) ck(cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking), "stream");
    for (int i = 0; i < 2 && s == FDK_OK; i++)
        ck(cudaEventCreateWithFlags(&h->sync_ev[i], cudaEventDisableTiming), "event");
    if (s == FDK_OK) ck(cudaHostAlloc((void **)&h->h_word, sizeof(unsigned int), 0), "pinned word");
    // geometry tables (FP64 -> FP32)
    std::vector<double> H(W);
    std::vector<float> cos(g->nu * g->nv);
    h->mats.resize(12 * g->n_proj);
    if (s == FDK_OK) s = fdk_filter_design(g->filter_type, g->nu, 1, H.data(), W);
    if (s == FDK_OK) s = fdk_cos_table(g, cos.data());
    if (s == FDK_OK) s = fdk_projection_matrices(g, nullptr, h->mats.data());
    if (s == FDK_OK) s = h->tables.create(H.data(), (int)W);
    const long long frame = g->nu * g->nv;
    if (s == FDK_OK) ck(cudaMalloc(&h->d_cos, sizeof(float) * frame), "cos table");
    if (s == FDK_OK)
        ck(cudaMemcpyAsync(h->d_cos, cos.data(), sizeof(float) * frame, cudaMemcpyHostToDevice, h->compute),
           "cos copy");
    if (s == FDK_OK) ck(cudaMalloc(&h->d_mats, sizeof(float) * h->mats.size()), "matrices");
    if (s == FDK_OK)
        ck(cudaMemcpyAsync(h->d_mats, h->mats.data(), sizeof(float) * h->mats.size(), cudaMemcpyHostToDevice,
                           h->compute),
           "matrices");
    h->chunk = std::min(batch, 32);
    const int n_slots = (batch + h->chunk - 1) / h->chunk + 2;
    h->d_raw.assign(n_slots, nullptr);
    h->raw_ready.assign(n_slots, nullptr);
    h->raw_free.assign(n_slots, nullptr);
    for (int i = 0; i < n_slots && s == FDK_OK; i++) {
        ck(cudaMalloc(&h->d_raw[i], sizeof(float) * frame * h->chunk), "raw views");
        ck(cudaEventCreateWithFlags(&h->raw_ready[i], cudaEventDisableTiming), "event");
        ck(cudaEventCreateWithFlags(&h->raw_free[i], cudaEventDisableTiming), "event");
    }
    const size_t esz = h->layout == FDK_LAYOUT_MIRROR ? (h->dtype == FDK_DTYPE_F16 ? 4 : 8) : 4;
    for (int i = 0; i < 2 && s == FDK_OK; i++)
        ck(cudaMalloc(&h->d_filt[i], esz * frame * batch), "filtered views");
    if (s == FDK_OK) ck(cudaMalloc(&h->d_overflow, sizeof(unsigned int)), "overflow flag");
    if (s == FDK_OK) ck(cudaMemsetAsync(h->d_overflow, 0, sizeof(unsigned int), h->compute), "overflow flag");
    if (s == FDK_OK) ck(cudaEventCreateWithFlags(&h->done, cudaEventDisableTiming), "event");
    if (s == FDK_OK && h->dtype == FDK_DTYPE_F16) {
        // FP16 views hold the filtered values divided by the cosine table's SOD^2 * AAF factor
        // (raw line-integral units); the backprojection multiplies it back.
        double aaf = 0;
        s = fdk_angular_ramp_factor(g, &aaf);
        const float k = (float)(g->sod * g->sod * aaf);
        h->out_scale = 1.0f / k;
        if (s == FDK_OK) ck(cudaMalloc(&h->d_scale, sizeof(float)), "scale");
        if (s == FDK_OK)
            ck(cudaMemcpyAsync(h->d_scale, &k, sizeof(float), cudaMemcpyHostToDevice, h->compute), "scale");
        // the filter, chosen by measurement: on the C3/C4 workloads the split-FP16 tensor-core
        // GEMM (fdk_toeplitz_*) matches the FFT filter's accuracy (rel-L2 2e-4, the FP16 output
        // rounding) in 0.61x (C3) / 0.67x (C4) of its time.  The FFT filter remains where the GEMM
        // cannot run (nu not a multiple of 256, nv of 128) or when FDK_FILTER=fft.
        const char *want = std::getenv("FDK_FILTER");
        const bool fft_only = want && std::string(want) == "fft";
        if (s == FDK_OK && !fft_only && g->nu % 256 == 0 && g->nv % 128 == 0) {
            const int rc = fdk_toeplitz_create(&h->tpz, cos.data(), H.data(), g->nu, g->nv, W, h->pad, 0, 1,
                                               h->out_scale, device);
            if (rc != FDK_OK) {
                h->tpz = nullptr;  // e.g. not an sm_100 GPU: the FFT filter serves
                clear_error();
            }
        }
    }
    if (s == FDK_OK) {
        const uint64_t d = (uint64_t)depth, z0 = (uint64_t)top_z;
        fdk_box top{0, 0, z0, (uint64_t)g->nx, (uint64_t)g->ny, d};
        fdk_box bot{0, 0, (uint64_t)g->nz - z0 - d, (uint64_t)g->nx, (uint64_t)g->ny, d};
        // the reconstructor feeds the handle device-resident views only (no host-view staging:
        // a view count of 1 keeps those buffers minimal)
        s = fdk_bp_create(&h->bp, (int)g->nv, (int)g->nu, 1, (int)g->nx, (int)g->ny, (int)g->nz, &top, &bot,
                          precision, device);
        if (s == FDK_OK && h->d_scale) s = fdk_bp_set_acc_scale_internal(h->bp, h->d_scale);
        // the quarter-turn kernel where the scan and the grid have the symmetry
        if (s == FDK_OK) s = fdk_bp_sym_setup_internal(h->bp, h->mats.data(), (int)g->n_proj, &h->sym_rot);
        // MIXED: the staged kernel reads each batch converted to the interpolation layout
        if (s == FDK_OK && precision == FDK_BP_MIXED) s = fdk_bp_reserve_lerp_internal(h->bp, h->batch);
        if (s == FDK_OK && precision == FDK_BP_MIXED)
            s = fdk_bp_choose_lerp_box_internal(h->bp, h->mats.data(), (int)g->n_proj);
    }
    if (s == FDK_OK) s = wait_stream(h->compute, h->sync_ev[0], "fdk_recon_create");  // set-up copies landed
    if (s != FDK_OK) {
        recon_release(h);
        return s;
    }
    *out = h;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_recon_push(fdk_recon *h, const float *host_views, int64_t first, int64_t n) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && host_views, "NULL argument");
    FDK_CHECK_ARG(first >= 0 && n > 0 && first + n <= h->g.n_proj, "view range [%lld, %lld) outside 0..%lld",
                  (long long)first, (long long)(first + n), (long long)h->g.n_proj);
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    const std::vector<int64_t> ids = consecutive(first, n);
    return push_host(h, host_views, ids.data(), n);
    FDK_ABI_END
}

int fdk_recon_push_views(fdk_recon *h, const float *host_views, const int64_t *views, int64_t n) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && host_views && views && n > 0, "NULL argument or empty list");
    FDK_TRY(check_ids(h, views, n));
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    return push_host(h, host_views, views, n);
    FDK_ABI_END
}

int fdk_recon_push_folder(fdk_recon *h, const char *folder, int64_t first, int64_t n, int32_t step, int32_t start,
                          int32_t threads) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && folder, "NULL argument");
    FDK_CHECK_ARG(first >= 0 && n > 0 && first + n <= h->g.n_proj, "view range [%lld, %lld) outside 0..%lld",
                  (long long)first, (long long)(first + n), (long long)h->g.n_proj);
    FDK_CHECK_ARG(step >= 1 && start >= 0, "step %d / start %d", step, start);
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    const int nu = (int)h->g.nu, nv = (int)h->g.nv;
    const long long frame = (long long)nu * nv;
    const int cap = h->chunk;
    // sizes of every file first, as the reference's folder loader
    for (long long i = 0; i < n; i++) {
        const std::string p = proj_file_path(folder, (first + i) * step + start);
        FILE *fp = std::fopen(p.c_str(), "rb");
        long long sz = -1;
        if (fp) {
            std::fseek(fp, 0, SEEK_END);
            sz = std::ftell(fp);
            std::fclose(fp);
        }
        if (sz != frame * (long long)sizeof(float)) {
            set_error("%s: %s (expected %lld bytes of FP32, %d x %d)", p.c_str(), sz < 0 ? "missing" : "wrong size",
                      frame * (long long)sizeof(float), nu, nv);
            return FDK_ERR_IO;
        }
    }
    for (int k = 0; k < 2; k++) {
        if (!h->h_stage[k]) FDK_CUDA(cudaHostAlloc((void **)&h->h_stage[k], sizeof(float) * frame * cap, 0));
        if (!h->stage_free[k]) {
            FDK_CUDA(cudaEventCreateWithFlags(&h->stage_free[k], cudaEventDisableTiming));
            FDK_CUDA(cudaEventRecord(h->stage_free[k], h->copy));
        }
    }
    int b = 0;
    for (long long c = 0; c < n; c += cap, b ^= 1) {
        const int m = (int)std::min<long long>(cap, n - c);
        FDK_TRY(wait_event(h->stage_free[b], "staging copy"));  // staging b's previous copy has landed
        FDK_TRY(read_views(folder, nu, nv, first + c, m, step, start, h->h_stage[b], threads));
        const int k = h->slot;
        h->slot = (k + 1) % (int)h->d_raw.size();
        FDK_CUDA(cudaStreamWaitEvent(h->copy, h->raw_free[k], 0));
        FDK_CUDA(cudaMemcpyAsync(h->d_raw[k], h->h_stage[b], sizeof(float) * frame * m, cudaMemcpyHostToDevice,
                                 h->copy));
        FDK_CUDA(cudaEventRecord(h->stage_free[b], h->copy));
        FDK_CUDA(cudaEventRecord(h->raw_ready[k], h->copy));
        FDK_CUDA(cudaStreamWaitEvent(h->compute, h->raw_ready[k], 0));
        const std::vector<int64_t> ids = consecutive(first + c, m);
        FDK_TRY(process_chunk(h, h->d_raw[k], ids.data(), m, h->raw_free[k], true));
    }
    return FDK_OK;
    FDK_ABI_END
}

// Device views: filtered straight from the caller's memory, batch by batch.
int push_device_ids(fdk_recon *h, const float *dev_views, const int64_t *ids, int64_t n) {
    const long long frame = h->g.nu * h->g.nv;
    const int cap = h->precision == FDK_BP_FP32_EXACT ? std::min(h->batch, 32) : h->batch;
    for (long long c = 0; c < n; c += cap) {
        const int m = (int)std::min<long long>(cap, n - c);
        FDK_TRY(process_chunk(h, dev_views + c * frame, ids + c, m, nullptr, false));
    }
    return FDK_OK;
}

int fdk_recon_push_device(fdk_recon *h, const float *dev_views, int64_t first, int64_t n) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && dev_views, "NULL argument");
    FDK_CHECK_ARG(first >= 0 && n > 0 && first + n <= h->g.n_proj, "view range outside the scan");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    const std::vector<int64_t> ids = consecutive(first, n);
    return push_device_ids(h, dev_views, ids.data(), n);
    FDK_ABI_END
}

int fdk_recon_push_device_views(fdk_recon *h, const float *dev_views, const int64_t *views, int64_t n) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && dev_views && views && n > 0, "NULL argument or empty list");
    FDK_TRY(check_ids(h, views, n));
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    return push_device_ids(h, dev_views, views, n);
    FDK_ABI_END
}

int fdk_recon_filter_kind(fdk_recon *h, int32_t *kind) {
    FDK_CHECK_ARG(h && kind, "NULL argument");
    *kind = h->tpz ? 1 : 0;
    return FDK_OK;
}

int fdk_recon_bp_kernel(fdk_recon *h, int32_t *kind) {
    FDK_CHECK_ARG(h && kind, "NULL argument");
    *kind = h->precision == FDK_BP_FP32_EXACT ? 0 : (h->sym_rot ? 2 : 1);
    return FDK_OK;
}

int fdk_recon_flush(fdk_recon *h) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    return flush_all(h);
    FDK_ABI_END
}

int fdk_recon_sync(fdk_recon *h, int64_t timeout_ms) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(flush_all(h));
    FDK_CUDA(cudaEventRecord(h->done, h->compute));
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t limit = timeout_ms > 0 ? timeout_ms : 600000;
    for (;;) {
        cudaError_t e = cudaEventQuery(h->done);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_status(e, "fdk_recon_sync", __FILE__, __LINE__);
        const auto el = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0);
        if (el.count() > limit) return fail(FDK_ERR_TIMEOUT, "fdk_recon_sync: work not finished after %lld ms",
                                            (long long)limit);
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    FDK_CUDA(cudaMemcpyAsync(h->h_word, h->d_overflow, sizeof(unsigned int), cudaMemcpyDeviceToHost, h->compute));
    FDK_TRY(wait_stream(h->compute, h->sync_ev[0], "overflow flag"));
    const unsigned int ovf = *h->h_word;
    if (ovf)
        return fail(FDK_ERR_DEVICE_CHECK, "filtered views exceeded the FP16 range; use FDK_BP_FP32 for this data");
    if (h->tpz) FDK_TRY(fdk_toeplitz_check(h->tpz));
    return fdk_bp_check_internal(h->bp);  // a backprojection wait that ran out on the device
    FDK_ABI_END
}

int fdk_recon_get_volume(fdk_recon *h, float *host_vol, int64_t size) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h && host_vol, "NULL argument");
    {
        DeviceGuard dg(h->device);
        FDK_TRY(dg.status);
        FDK_TRY(flush_all(h));
    }
    // band by band, overlapping the last batch's backprojection; then the filter checks
    FDK_TRY(fdk_bp_get_volume(h->bp, host_vol, size));
    return fdk_recon_sync(h, 0);
    FDK_ABI_END
}

int fdk_recon_sample(fdk_recon *h, const int32_t *host_xyz, int64_t n, float *host_out) {
    FDK_ABI_BEGIN
    clear_error();
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    FDK_TRY(fdk_recon_sync(h, 0));
    return fdk_bp_sample(h->bp, host_xyz, n, host_out);
    FDK_ABI_END
}

int fdk_recon_stats(fdk_recon *h, double *bp_ms, double *filter_ms, int64_t *views) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(collect_filter_timers(h));
    int64_t cnt = 0;
    double ms = 0;
    FDK_TRY(fdk_bp_stats(h->bp, &cnt, &ms));
    if (bp_ms) *bp_ms = ms;
    if (filter_ms) *filter_ms = h->filter_ms;
    if (views) *views = h->views;
    return FDK_OK;
    FDK_ABI_END
}

int fdk_recon_launch_count(fdk_recon *h, int64_t *count) {
    FDK_CHECK_ARG(h && count, "NULL argument");
    *count = h->filter_launches + fdk_bp_launches_internal(h->bp);
    return FDK_OK;
}

int fdk_recon_reset(fdk_recon *h) {
    FDK_ABI_BEGIN
    FDK_CHECK_ARG(h != nullptr, "NULL handle");
    DeviceGuard dg(h->device);
    FDK_TRY(dg.status);
    FDK_TRY(wait_stream(h->copy, h->sync_ev[1], "fdk_recon_reset"));
    FDK_TRY(wait_stream(h->compute, h->sync_ev[0], "fdk_recon_reset"));
    FDK_TRY(collect_filter_timers(h));
    FDK_CUDA(cudaMemsetAsync(h->d_overflow, 0, sizeof(unsigned int), h->compute));
    h->filter_ms = 0;
    h->views = 0;
    h->filter_launches = 0;
    h->pending = 0;  // filtered views not yet backprojected are dropped with the volume
    h->held = false;
    h->ramp = 0;
    h->bviews[0].clear();
    h->bviews[1].clear();
    h->cur = 0;
    return fdk_bp_reset(h->bp);
    FDK_ABI_END
}

int fdk_recon_destroy(fdk_recon *h) { return recon_release(h); }

}  // extern "C"
