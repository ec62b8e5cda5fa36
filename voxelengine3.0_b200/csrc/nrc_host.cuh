// nrc_host.cuh — host side of the learned radiance cache (part of the
// render.cu translation unit): parameter storage, initialisation, the C ABI
// of include/ve.h, and the enqueue helpers the frame sequence calls.
#pragma once
#include <cmath>

struct ve_nrc {
    ve_ctx* c = nullptr;
    ve_nrc_config cfg{};
    ve::nrc::Grid grid{};
    size_t n_table = 0;  // feature pairs (levels x T)
    ve::DevBuf<float2> tp, tm, tv, tg;
    ve::DevBuf<uint32_t> th;
    ve::DevBuf<float> w, wm, wv, wg;
    ve::DevBuf<uint8_t> wimg;
    ve::DevBuf<ve::nrc::AdamState> adam;
    ve::DevBuf<float> loss;
    ve::DevBuf<uint32_t> status, nvalid;
    ve::DevBuf<float4> val;  // per validation cell: {mean target, samples}, {mean prediction}
    // host-API staging
    ve::DevBuf<ve::nrc::QRec> q;
    ve::DevBuf<ve::nrc::TRec> tr;
    ve::DevBuf<float4> out;
    // learned-frame buffers: queries (paths terminated at vertex 1) and
    // training samples
    ve::DevBuf<ve::nrc::QRec> fq, fs;
    ve::DevBuf<float4> fstage;   // per query: the path state its deposit needs (3 x float4)
    ve::DevBuf<uint8_t> fx, x;   // encoded input tiles (frames, host API)
    ve::DevBuf<ve::nrc::TRec> ftr;
    int grid_infer = 0, grid_train = 0;
    uint64_t trained_steps = 0;
    float last_loss = 0.0f;
};

namespace ve {
namespace nrc {

constexpr uint32_t kValCellsLog2 = 20;
// training steps after which cells without validation samples use the network
constexpr uint64_t kReadySteps = 16;

static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static float uniform(uint64_t& s, float lo, float hi) {
    return lo + (hi - lo) * float(double(splitmix(s) >> 11) * (1.0 / 9007199254740992.0));
}

static Grid make_grid(const ve_nrc_config& cfg) {
    Grid g{};
    g.log2T = cfg.log2_table;
    const double b = std::exp((std::log(double(cfg.max_resolution)) - std::log(double(cfg.base_resolution))) /
                              double(kLevels - 1));
    const double T = std::ldexp(1.0, int(cfg.log2_table));
    for (uint32_t l = 0; l < kLevels; l++) {
        const uint32_t r = uint32_t(std::floor(double(cfg.base_resolution) * std::pow(b, double(l)) + 1e-9));
        g.res[l] = std::max(r, 1u);
        const double v = double(g.res[l] + 1u);
        if (v * v * v <= T) g.dense_mask |= 1u << l;
    }
    return g;
}

static int launch_train(ve_nrc* m, cudaStream_t st, const QRec* q, const TRec* tr, const uint32_t* count, uint32_t n,
                        float inv_norm) {
    Args a{};
    a.q = q;
    a.tr = tr;
    a.count = count;
    a.n = n;
    a.table = m->th.p;
    a.wimg = reinterpret_cast<const uint4*>(m->wimg.p);
    a.grid = m->grid;
    a.wgrad = m->wg.p;
    a.tgrad = reinterpret_cast<float*>(m->tg.p);
    a.loss = m->loss.p;
    a.val = m->val.p;
    a.val_mask = (1u << kValCellsLog2) - 1u;
    a.inv_norm = inv_norm;
    a.status = m->status.p;
    a.nvalid = m->nvalid.p;
    k_nrc_mlp<true><<<m->grid_train, 128, kSmemTrain, st>>>(a);
    return VE_OK;
}

static Args infer_args(ve_nrc* m, const QRec* q, const uint32_t* count, uint32_t n) {
    Args a{};
    a.q = q;
    a.count = count;
    a.n = n;
    a.table = m->th.p;
    a.wimg = reinterpret_cast<const uint4*>(m->wimg.p);
    a.grid = m->grid;
    a.status = m->status.p;
    return a;
}

// Inference over `count` (device) or n rows: encode (+ stage), then the MLP
// with the epilogue `epi` (X holds n rows rounded up to whole tiles).
template <class Pre, class Epi>
static void launch_infer(ve_nrc* m, cudaStream_t st, const Args& a, uint8_t* X, Pre pre, Epi epi) {
    k_nrc_encode<Pre><<<m->c->num_sms * 8, 256, 0, st>>>(a, X, pre);
    k_nrc_infer<Epi><<<m->grid_infer, 128 * kInferGroups, kSmemInfer, st>>>(a, X, epi);
}

template <class Epi>
static int set_infer_attributes() {
    if (cudaFuncSetAttribute(k_nrc_infer<Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemInfer)) !=
        cudaSuccess)
        return VE_ERR_CUDA;
    cudaFuncSetAttribute(k_nrc_infer<Epi>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    return VE_OK;
}

static void launch_adam(ve_nrc* m, cudaStream_t st) {
    k_nrc_step<<<1, 1, 0, st>>>(m->adam.p, m->cfg.beta1, m->cfg.beta2);
    AdamArgs aa{m->cfg.learning_rate, m->cfg.beta1, m->cfg.beta2, m->cfg.eps, m->adam.p};
    k_nrc_adam_weights<<<(kWParams + 255) / 256, 256, 0, st>>>(m->w.p, m->wm.p, m->wv.p, m->wg.p, m->wimg.p, aa);
    k_nrc_adam_table<<<m->c->num_sms * 8, 256, 0, st>>>(m->tp.p, m->tm.p, m->tv.p, m->tg.p, m->th.p, m->n_table, aa);
}

static void enqueue_zero_grads(ve_nrc* m, cudaStream_t st) {
    cudaMemsetAsync(m->wg.p, 0, sizeof(float) * kWParams, st);
    cudaMemsetAsync(m->tg.p, 0, sizeof(float2) * m->n_table, st);
    cudaMemsetAsync(m->loss.p, 0, sizeof(float), st);
    cudaMemsetAsync(m->nvalid.p, 0, sizeof(uint32_t), st);
}
static int zero_grads(ve_nrc* m, cudaStream_t st) {
    enqueue_zero_grads(m, st);
    VE_CUDA(cudaGetLastError());
    return VE_OK;
}

// Frame buffers of a learned frame: queries and predictions for every path,
// the per-frame training sample set.  Returns whether a buffer moved.
static int prepare_frame(ve_nrc* m, uint64_t paths, bool* moved) {
    const void* before[] = {m->fq.p, m->fx.p, m->fstage.p, m->fs.p, m->ftr.p};
    int rc;
    if ((rc = m->fq.ensure(paths)) || (rc = m->fx.ensure(size_t((paths + kRows - 1) / kRows) * kTileBytes)) ||
        (rc = m->fstage.ensure(3 * paths)) || (rc = m->fs.ensure(m->cfg.train_samples)) ||
        (rc = m->ftr.ensure(m->cfg.train_samples)))
        return rc;
    const void* after[] = {m->fq.p, m->fx.p, m->fstage.p, m->fs.p, m->ftr.p};
    for (int i = 0; i < 5; i++) *moved |= before[i] != after[i];
    return VE_OK;
}

static int check_status(ve_nrc* m) {
    uint32_t s = 0;
    VE_CUDA(cudaMemcpyAsync(&s, m->status.p, 4, cudaMemcpyDeviceToHost, m->c->stream));
    VE_CUDA(cudaStreamSynchronize(m->c->stream));
    if (s) return fail(VE_ERR_CUDA, "learned cache: a tensor-core wait timed out");
    return VE_OK;
}

static int stage_inputs(ve_nrc* m, const ve_nrc_input* in, const float* target, uint32_t n) {
    static_assert(sizeof(ve_nrc_input) == sizeof(QRec), "ve_nrc_input mirrors the device record");
    int rc;
    if ((rc = m->q.ensure(n)) || (target && (rc = m->tr.ensure(n)))) return rc;
    cudaStream_t st = m->c->stream;
    VE_CUDA(cudaMemcpyAsync(m->q.p, in, sizeof(QRec) * n, cudaMemcpyHostToDevice, st));
    if (target) {
        std::vector<TRec> t(n);
        for (uint32_t i = 0; i < n; i++) {
            t[i] = TRec{};
            t[i].tr = target[3 * i];
            t[i].tg = target[3 * i + 1];
            t[i].tb = target[3 * i + 2];
            t[i].valid = 1u;
            t[i].cell = 0xFFFFFFFFu;
        }
        VE_CUDA(cudaMemcpyAsync(m->tr.p, t.data(), sizeof(TRec) * n, cudaMemcpyHostToDevice, st));
        VE_CUDA(cudaStreamSynchronize(st));
    }
    return VE_OK;
}

}  // namespace nrc
}  // namespace ve

extern "C" {

int ve_nrc_create(ve_ctx* c, const ve_nrc_config* cfg, ve_nrc** out) {
    using namespace ve;
    using namespace ve::nrc;
    if (!c || !cfg || !out) return fail(VE_ERR_INVALID, "nrc_create: null argument");
    if (cfg->log2_table < 8 || cfg->log2_table > 24 || cfg->base_resolution < 2 ||
        cfg->max_resolution < cfg->base_resolution || cfg->max_resolution > 65536 || cfg->train_samples == 0 ||
        cfg->train_samples > (1u << 22) || !(cfg->learning_rate > 0.0f) || !(cfg->beta1 >= 0.0f && cfg->beta1 < 1.0f) ||
        !(cfg->beta2 >= 0.0f && cfg->beta2 < 1.0f) || !(cfg->eps > 0.0f))
        return fail(VE_ERR_INVALID, "nrc_create: configuration out of range");
    cudaSetDevice(c->device);
    ve_nrc* m = new ve_nrc();
    m->c = c;
    m->cfg = *cfg;
    m->grid = make_grid(*cfg);
    m->n_table = size_t(kLevels) << cfg->log2_table;
    int rc;
    if ((rc = m->tp.ensure(m->n_table)) || (rc = m->tm.ensure(m->n_table)) || (rc = m->tv.ensure(m->n_table)) ||
        (rc = m->tg.ensure(m->n_table)) || (rc = m->th.ensure(m->n_table)) || (rc = m->w.ensure(kWParams)) ||
        (rc = m->wm.ensure(kWParams)) || (rc = m->wv.ensure(kWParams)) || (rc = m->wg.ensure(kWParams)) ||
        (rc = m->wimg.ensure(kWImage)) || (rc = m->adam.ensure(1)) || (rc = m->loss.ensure(1)) ||
        (rc = m->status.ensure(1)) || (rc = m->nvalid.ensure(1)) ||
        (rc = m->val.ensure(size_t(2) << kValCellsLog2))) {
        ve_nrc_destroy(m);
        return rc;
    }
    // initial parameters: uniform(+-sqrt(6 / 64)) hidden weights, a small
    // output layer, table features uniform(+-1e-4)
    std::vector<float> w(kWParams, 0.0f);
    uint64_t s = cfg->seed ^ 0x4E5243ull;
    for (uint32_t l = 0; l < kLayers; l++) {
        const float lim = l + 1u < kLayers ? std::sqrt(6.0f / 64.0f) : 0.1f * std::sqrt(6.0f / 64.0f);
        const uint32_t rows = l + 1u < kLayers ? 64u : kOutRows;
        for (uint32_t o = 0; o < rows; o++)
            for (uint32_t i = 0; i < kWidth; i++) w[(l * kWidth + o) * kWidth + i] = uniform(s, -lim, lim);
    }
    std::vector<float2> t(m->n_table);
    for (auto& e : t) e = make_float2(uniform(s, -1e-4f, 1e-4f), uniform(s, -1e-4f, 1e-4f));
    rc = ve_nrc_set_params(m, w.data(), reinterpret_cast<const float*>(t.data()));
    if (rc) {
        ve_nrc_destroy(m);
        return rc;
    }
    static_assert(kSmemTrain <= 227u * 1024u, "training tile set exceeds shared memory");
    if (cudaFuncSetAttribute(k_nrc_mlp<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemTrain)) !=
            cudaSuccess ||
        set_infer_attributes<StoreOut>() != VE_OK || set_frame_infer_attributes() != VE_OK) {
        ve_nrc_destroy(m);
        return fail(VE_ERR_CUDA, "nrc_create: shared-memory attribute refused");
    }
    c->nrcs.push_back(m);
    int occ_i = 0, occ_t = 0;
    // resident inference CTAs per SM: shared memory (the kernel prefers the
    // largest carveout) and 512 tensor-memory columns, 128 per CTA; the
    // occupancy query is taken as a floor only, since it assumes the default
    // carveout
    cudaFuncSetAttribute(k_nrc_mlp<true>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_i, k_nrc_infer<StoreOut>, 128 * kInferGroups,
                                                      kSmemInfer) != cudaSuccess)
        occ_i = 1;
    int smem_sm = 0;
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
    const int by_smem = smem_sm / int(kSmemInfer + 2048u);
    occ_i = std::max(1, std::min(std::max(occ_i, by_smem), std::min(3, int(512 / kTmemInfer))));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, k_nrc_mlp<true>, 128, kSmemTrain);
    cudaGetLastError();
    occ_t = 1;
    m->grid_infer = c->num_sms * occ_i;
    m->grid_train = c->num_sms * occ_t;
    *out = m;
    return VE_OK;
}

int ve_nrc_destroy(ve_nrc* m) {
    if (!m) return VE_OK;
    cudaSetDevice(m->c->device);
    cudaStreamSynchronize(m->c->stream);
    for (auto& sl : m->c->scenes)
        if (sl.nrc == m) sl.nrc = nullptr;
    auto& v = m->c->nrcs;
    v.erase(std::remove(v.begin(), v.end(), m), v.end());
    for (auto* b : {&m->tp, &m->tm, &m->tv, &m->tg}) b->release();
    m->fstage.release();
    m->fx.release();
    m->x.release();
    m->th.release();
    for (auto* b : {&m->w, &m->wm, &m->wv, &m->wg, &m->loss}) b->release();
    m->val.release();
    m->wimg.release();
    m->adam.release();
    m->status.release();
    m->nvalid.release();
    m->q.release();
    m->tr.release();
    m->out.release();
    m->fq.release();
    m->fs.release();
    m->ftr.release();
    delete m;
    return VE_OK;
}

int ve_nrc_param_counts(const ve_nrc* m, uint64_t* n_weights, uint64_t* n_table) {
    using namespace ve;
    if (!m || !n_weights || !n_table) return fail(VE_ERR_INVALID, "nrc_param_counts: null argument");
    *n_weights = nrc::kWParams;
    *n_table = 2ull * m->n_table;
    return VE_OK;
}

int ve_nrc_get_params(ve_nrc* m, float* weights, float* table) {
    using namespace ve;
    if (!m) return fail(VE_ERR_INVALID, "nrc_get_params: null handle");
    cudaSetDevice(m->c->device);
    VE_CUDA(cudaStreamSynchronize(m->c->stream));
    // the context's stream is non-blocking: every copy goes through it
    if (weights)
        VE_CUDA(cudaMemcpyAsync(weights, m->w.p, sizeof(float) * nrc::kWParams, cudaMemcpyDeviceToHost, m->c->stream));
    if (table)
        VE_CUDA(cudaMemcpyAsync(table, m->tp.p, sizeof(float2) * m->n_table, cudaMemcpyDeviceToHost, m->c->stream));
    VE_CUDA(cudaStreamSynchronize(m->c->stream));
    return VE_OK;
}

int ve_nrc_set_params(ve_nrc* m, const float* weights, const float* table) {
    using namespace ve;
    using namespace ve::nrc;
    if (!m) return fail(VE_ERR_INVALID, "nrc_set_params: null handle");
    cudaSetDevice(m->c->device);
    cudaStream_t st = m->c->stream;
    VE_CUDA(cudaStreamSynchronize(st));
    if (weights) {
        // on the context's (non-blocking) stream, so the kernels below see the
        // whole copy: a legacy-stream copy from pageable memory may return
        // before its DMA has landed
        VE_CUDA(cudaMemcpyAsync(m->w.p, weights, sizeof(float) * kWParams, cudaMemcpyHostToDevice, st));
        VE_CUDA(cudaMemsetAsync(m->wimg.p, 0, kWImage, st));
        k_nrc_weights_image<<<(kWParams + 255) / 256, 256, 0, st>>>(m->w.p, m->wimg.p);
    }
    if (table) {
        VE_CUDA(cudaMemcpyAsync(m->tp.p, table, sizeof(float2) * m->n_table, cudaMemcpyHostToDevice, st));
        k_nrc_table_half<<<m->c->num_sms * 8, 256, 0, st>>>(m->tp.p, m->th.p, m->n_table);
    }
    // a new parameter set restarts the optimiser
    VE_CUDA(cudaMemsetAsync(m->wm.p, 0, sizeof(float) * kWParams, st));
    VE_CUDA(cudaMemsetAsync(m->wv.p, 0, sizeof(float) * kWParams, st));
    VE_CUDA(cudaMemsetAsync(m->wg.p, 0, sizeof(float) * kWParams, st));
    VE_CUDA(cudaMemsetAsync(m->tm.p, 0, sizeof(float2) * m->n_table, st));
    VE_CUDA(cudaMemsetAsync(m->tv.p, 0, sizeof(float2) * m->n_table, st));
    VE_CUDA(cudaMemsetAsync(m->tg.p, 0, sizeof(float2) * m->n_table, st));
    VE_CUDA(cudaMemsetAsync(m->adam.p, 0, sizeof(AdamState), st));
    VE_CUDA(cudaMemsetAsync(m->status.p, 0, 4, st));
    VE_CUDA(cudaMemsetAsync(m->val.p, 0, sizeof(float4) * (size_t(2) << kValCellsLog2), st));
    VE_CUDA(cudaStreamSynchronize(st));
    m->trained_steps = 0;
    return VE_OK;
}

int ve_nrc_infer(ve_nrc* m, const ve_nrc_input* in, uint32_t n, float* rgb) {
    using namespace ve;
    if (!m || (!in && n) || (!rgb && n)) return fail(VE_ERR_INVALID, "nrc_infer: null argument");
    if (n == 0) return VE_OK;
    cudaSetDevice(m->c->device);
    int rc;
    if ((rc = nrc::stage_inputs(m, in, nullptr, n)) || (rc = m->out.ensure(n))) return rc;
    cudaStream_t st = m->c->stream;
    if ((rc = m->x.ensure(size_t((n + nrc::kRows - 1) / nrc::kRows) * nrc::kTileBytes))) return rc;
    nrc::launch_infer(m, st, nrc::infer_args(m, m->q.p, nullptr, n), m->x.p, nrc::NoStage{}, nrc::StoreOut{m->out.p});
    std::vector<float4> o(n);
    VE_CUDA(cudaMemcpyAsync(o.data(), m->out.p, sizeof(float4) * n, cudaMemcpyDeviceToHost, st));
    VE_CUDA(cudaStreamSynchronize(st));
    if ((rc = nrc::check_status(m))) return rc;
    for (uint32_t i = 0; i < n; i++) {
        rgb[3 * i] = o[i].x;
        rgb[3 * i + 1] = o[i].y;
        rgb[3 * i + 2] = o[i].z;
    }
    return VE_OK;
}

int ve_nrc_gradients(ve_nrc* m, const ve_nrc_input* in, const float* target, uint32_t n, float* weight_grad,
                     float* table_grad, float* loss) {
    using namespace ve;
    if (!m || !in || !target || n == 0) return fail(VE_ERR_INVALID, "nrc_gradients: null argument or no samples");
    cudaSetDevice(m->c->device);
    cudaStream_t st = m->c->stream;
    int rc;
    if ((rc = nrc::stage_inputs(m, in, target, n)) || (rc = nrc::zero_grads(m, st))) return rc;
    nrc::launch_train(m, st, m->q.p, m->tr.p, nullptr, n, 1.0f / (3.0f * float(n)));
    float l = 0.0f;
    if (weight_grad)
        VE_CUDA(cudaMemcpyAsync(weight_grad, m->wg.p, sizeof(float) * nrc::kWParams, cudaMemcpyDeviceToHost, st));
    if (table_grad)
        VE_CUDA(cudaMemcpyAsync(table_grad, m->tg.p, sizeof(float2) * m->n_table, cudaMemcpyDeviceToHost, st));
    VE_CUDA(cudaMemcpyAsync(&l, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    VE_CUDA(cudaStreamSynchronize(st));
    if ((rc = nrc::check_status(m))) return rc;
    // leave no stale gradient behind for the next optimiser step
    if ((rc = nrc::zero_grads(m, st))) return rc;
    VE_CUDA(cudaStreamSynchronize(st));
    if (loss) *loss = l / (3.0f * float(n));
    return VE_OK;
}

int ve_nrc_train(ve_nrc* m, const ve_nrc_input* in, const float* target, uint32_t n, float* loss) {
    using namespace ve;
    if (!m || !in || !target || n == 0) return fail(VE_ERR_INVALID, "nrc_train: null argument or no samples");
    cudaSetDevice(m->c->device);
    cudaStream_t st = m->c->stream;
    int rc;
    if ((rc = nrc::stage_inputs(m, in, target, n)) || (rc = nrc::zero_grads(m, st))) return rc;
    nrc::launch_train(m, st, m->q.p, m->tr.p, nullptr, n, 1.0f / (3.0f * float(n)));
    nrc::launch_adam(m, st);
    float l = 0.0f;
    VE_CUDA(cudaMemcpyAsync(&l, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    VE_CUDA(cudaStreamSynchronize(st));
    if ((rc = nrc::check_status(m))) return rc;
    m->trained_steps++;
    m->last_loss = l / (3.0f * float(n));
    if (loss) *loss = m->last_loss;
    return VE_OK;
}

int ve_nrc_stats(ve_nrc* m, float* loss, uint64_t* samples, uint64_t* steps) {
    using namespace ve;
    if (!m) return fail(VE_ERR_INVALID, "nrc_stats: null handle");
    cudaSetDevice(m->c->device);
    VE_CUDA(cudaStreamSynchronize(m->c->stream));
    float l = 0.0f;
    uint32_t n = 0;
    VE_CUDA(cudaMemcpyAsync(&l, m->loss.p, sizeof(float), cudaMemcpyDeviceToHost, m->c->stream));
    VE_CUDA(cudaMemcpyAsync(&n, m->nvalid.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, m->c->stream));
    VE_CUDA(cudaStreamSynchronize(m->c->stream));
    int rc;
    if ((rc = nrc::check_status(m))) return rc;
    if (loss) *loss = n ? l / (3.0f * float(n)) : 0.0f;
    if (samples) *samples = n;
    if (steps) *steps = m->trained_steps;
    return VE_OK;
}

int ve_scene_set_nrc(ve_ctx* c, int scene_id, ve_nrc* m) {
    if (c) ve::join_alt(c);  // after the second frame set's frames in flight
    using namespace ve;
    if (!c) return fail(VE_ERR_INVALID, "scene_set_nrc: null context");
    if (scene_id < 0 || size_t(scene_id) >= c->scenes.size() || !c->scenes[scene_id].live)
        return fail(VE_ERR_NOT_FOUND, "scene_set_nrc: unknown scene");
    if (m && m->c != c) return fail(VE_ERR_INVALID, "scene_set_nrc: the learned cache belongs to another context");
    c->scenes[scene_id].nrc = m;
    return VE_OK;
}

}  // extern "C"
