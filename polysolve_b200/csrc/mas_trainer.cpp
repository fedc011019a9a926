// Host side of the warm-start network's GPU training: the mas_ws_trainer handle (storage of the
// samples, scratch, the training loop over the kernels of mas_ws_train.cu) and its C ABI. Sample
// collection from a solver is in mas_capi.cpp (it runs the solver's prediction pipeline).

#include "mas_trainer.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>

#include <cuda_runtime.h>

#include "polysolve_mas.h"

using namespace pmas;

namespace
{
    // Device address of a field of the device-resident training state.
    const double *state_field(const WsTrainState *st, size_t offset)
    {
        return reinterpret_cast<const double *>(reinterpret_cast<const char *>(st) + offset);
    }
} // namespace

mas_ws_trainer::~mas_ws_trainer()
{
    if (stream)
    {
        cudaSetDevice(device);
        cudaStreamSynchronize(stream);
        cudaStreamDestroy(stream);
    }
}

void mas_ws_trainer::init(const float *params, long long count)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    {
        cudaGetLastError();
        throw Error(ERR_NO_DEVICE, "No Nvidia GPU!!");
    }
    if (!params || count != WS_PARAMS)
        throw Error(ERR_INVALID, "[MAS] warm start trainer: expected " + std::to_string(WS_PARAMS) +
                                     " float32 initial parameters");
    for (long long i = 0; i < count; ++i)
        if (!std::isfinite(params[i]))
            throw Error(ERR_INVALID, "[MAS] warm start trainer: non-finite initial parameter");
    cuda_check(cudaGetDevice(&device), "get device");
    cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream create");
    prm.alloc(WS_PARAMS, "warm start trainer");
    adam_m.alloc(WS_PARAMS, "warm start trainer");
    adam_v.alloc(WS_PARAMS, "warm start trainer");
    grad.alloc(WS_PARAMS, "warm start trainer");
    wl.alloc((size_t)WS_LAYERS * WS_LAYER_WEIGHTS, "warm start trainer");
    st.alloc(1, "warm start trainer");
    cuda_check(cudaMemcpyAsync(prm.get(), params, sizeof(float) * WS_PARAMS, cudaMemcpyHostToDevice, stream),
               "upload parameters");
    cuda_check(cudaMemsetAsync(adam_m.get(), 0, adam_m.bytes(), stream), "memset");
    cuda_check(cudaMemsetAsync(adam_v.get(), 0, adam_v.bytes(), stream), "memset");
    cuda_check(cudaMemsetAsync(st.get(), 0, st.bytes(), stream), "memset");
    launch_tr_weights_bf16(prm.get(), wl.get(), stream);
    cuda_check(cudaStreamSynchronize(stream), "trainer init");
}

int mas_ws_trainer::pattern_for(const void *owner, uint64_t key, const BankedMatrix &A, const int *diag_slot,
                                cudaStream_t s)
{
    for (size_t i = patterns.size(); i-- > 0;)
        if (patterns[i]->owner == owner && patterns[i]->key == key && patterns[i]->banks == A.banks &&
            patterns[i]->slots == A.slots)
            return (int)i;
    auto p = std::make_unique<Pattern>();
    p->owner = owner;
    p->key = key;
    p->banks = A.banks;
    p->slots = A.slots;
    const size_t nodes = (size_t)A.banks * 32;
    const size_t entries = (size_t)std::max<long long>(A.slots, 1) * 32;
    p->slice.alloc((size_t)A.banks + 1, "warm start trainer pattern");
    p->rowlen.alloc(std::max<size_t>(nodes, 1), "warm start trainer pattern");
    p->cols.alloc(entries, "warm start trainer pattern");
    p->diag_slot.alloc(std::max<size_t>(nodes, 1), "warm start trainer pattern");
    p->mirror.alloc(entries, "warm start trainer pattern");
    p->real.alloc(std::max<size_t>(nodes, 1), "warm start trainer pattern");
    cuda_check(cudaMemcpyAsync(p->slice.get(), A.slice.get(), sizeof(long long) * ((size_t)A.banks + 1),
                               cudaMemcpyDeviceToDevice, s),
               "copy pattern");
    if (nodes)
    {
        cuda_check(cudaMemcpyAsync(p->rowlen.get(), A.rowlen.get(), sizeof(int) * nodes, cudaMemcpyDeviceToDevice, s),
                   "copy pattern");
        cuda_check(cudaMemcpyAsync(p->diag_slot.get(), diag_slot, sizeof(int) * nodes, cudaMemcpyDeviceToDevice, s),
                   "copy pattern");
    }
    if (A.slots > 0)
        cuda_check(cudaMemcpyAsync(p->cols.get(), A.cols.get(), sizeof(int) * (size_t)A.slots * 32,
                                   cudaMemcpyDeviceToDevice, s),
                   "copy pattern");
    launch_tr_pattern(A.view(), diag_slot, A.slots, p->mirror.get(), p->real.get(), s);
    patterns.push_back(std::move(p));
    return (int)patterns.size() - 1;
}

void mas_ws_trainer::add_sample(int pattern, const BankedMatrix &A, const float *wslot, const float *feat_raw,
                                const WsState *ws, const double *rg, const WsHistory &hist, const double *x_exact,
                                size_t len, cudaStream_t s)
{
    const Pattern &P = *patterns[pattern];
    const size_t nodes = (size_t)P.banks * 32;
    const size_t entries = (size_t)std::max<long long>(P.slots, 1) * 32;
    auto smp = std::make_unique<Sample>();
    smp->pattern = pattern;
    smp->vals32.alloc(entries * 9, "warm start trainer sample");
    smp->wslot.alloc(entries, "warm start trainer sample");
    smp->wT.alloc(entries, "warm start trainer sample");
    smp->feat.alloc(std::max<size_t>(nodes, 1) * WS_FEATURES, "warm start trainer sample");
    smp->re.alloc(std::max<size_t>(len, 1), "warm start trainer sample");
    smp->sc.alloc(2, "warm start trainer sample");
    const int capacity = 1024;
    coll_partials.alloc(capacity, "warm start trainer");
    coll_counter.alloc(1, "warm start trainer");
    launch_tr_sample(A.view(), P.slots, P.mirror.get(), P.real.get(), wslot, feat_raw, ws, rg, hist, x_exact, len,
                     smp->vals32.get(), smp->wslot.get(), smp->wT.get(), smp->feat.get(), smp->re.get(), smp->sc.get(),
                     coll_partials.get(), coll_counter.get(), capacity, s);
    samples.push_back(std::move(smp));
}

WsTrainView mas_ws_trainer::view(int i) const
{
    const Sample &S = *samples[i];
    const Pattern &P = *patterns[S.pattern];
    return WsTrainView{P.banks,         P.slice.get(),    P.rowlen.get(), P.cols.get(),
                       P.diag_slot.get(), P.real.get(),   S.vals32.get(), S.wslot.get(),
                       S.wT.get(),      S.feat.get(),     S.re.get(),     S.sc.get()};
}

void mas_ws_trainer::ensure_scratch(int nodes)
{
    if (nodes <= cap_nodes)
        return;
    const size_t n = (size_t)nodes, hid = n * WS_HIDDEN;
    z0.alloc(hid, "warm start trainer scratch");
    for (auto &b : z)
        b.alloc(hid, "warm start trainer scratch");
    for (auto &b : h)
        b.alloc(hid, "warm start trainer scratch");
    for (auto &b : m)
        b.alloc(hid, "warm start trainer scratch");
    gh.alloc(hid, "warm start trainer scratch");
    g1.alloc(hid, "warm start trainer scratch");
    gm.alloc(hid, "warm start trainer scratch");
    c.alloc(n * 3, "warm start trainer scratch");
    Ac.alloc(n * 3, "warm start trainer scratch");
    partials.alloc((size_t)ws_train_ctas(nodes) * WS_PARAMS, "warm start trainer scratch");
    red.alloc((size_t)2 * ((n / 32 + 7) / 8 + 1), "warm start trainer scratch");
    cap_nodes = nodes;
}

WsTrainScratch mas_ws_trainer::scratch()
{
    WsTrainScratch w{};
    w.z0 = z0.get();
    for (int l = 0; l < WS_LAYERS; ++l)
    {
        w.z[l] = z[l].get();
        w.m[l] = m[l].get();
    }
    for (int l = 0; l <= WS_LAYERS; ++l)
        w.h[l] = h[l].get();
    w.c = c.get();
    w.Ac = Ac.get();
    w.gh = gh.get();
    w.g1 = g1.get();
    w.gm = gm.get();
    w.partials = partials.get();
    w.red = red.get();
    w.st = st.get();
    return w;
}

void mas_ws_trainer::gradient(int i, float *out, double *loss)
{
    cuda_check(cudaSetDevice(device), "set device");
    if (i < 0 || i >= (int)samples.size())
        throw Error(ERR_INVALID, "[MAS] warm start trainer: no such sample");
    const WsTrainView S = view(i);
    ensure_scratch(S.banks * 32);
    const WsTrainScratch w = scratch();
    launch_tr_forward(S, prm.get(), wl.get(), w, stream);
    launch_tr_backward(S, prm.get(), wl.get(), w, grad.get(), stream);
    WsTrainState hs;
    cuda_check(cudaMemcpyAsync(&hs, st.get(), sizeof(hs), cudaMemcpyDeviceToHost, stream), "download");
    if (out)
        cuda_check(cudaMemcpyAsync(out, grad.get(), sizeof(float) * WS_PARAMS, cudaMemcpyDeviceToHost, stream),
                   "download");
    cuda_check(cudaStreamSynchronize(stream), "trainer gradient");
    if (loss)
        *loss = hs.loss;
}

void mas_ws_trainer::train(const int *idx, const float *lr, int count, double *loss_out)
{
    cuda_check(cudaSetDevice(device), "set device");
    for (int k = 0; k < count; ++k)
        if (idx[k] < 0 || idx[k] >= (int)samples.size() || !std::isfinite(lr[k]))
            throw Error(ERR_INVALID, "[MAS] warm start trainer: bad sample index or learning rate");
    int maxn = 0;
    for (int k = 0; k < count; ++k)
        maxn = std::max(maxn, view(idx[k]).banks * 32);
    ensure_scratch(maxn);
    losses.alloc(std::max(count, 1), "warm start trainer losses");
    const WsTrainScratch w = scratch();
    // The whole list runs without a host round trip; the losses are read once at the end.
    for (int k = 0; k < count; ++k)
    {
        const WsTrainView S = view(idx[k]);
        launch_tr_forward(S, prm.get(), wl.get(), w, stream);
        cuda_check(cudaMemcpyAsync(losses.get() + k, state_field(w.st, offsetof(WsTrainState, loss)), sizeof(double), cudaMemcpyDeviceToDevice, stream),
                   "loss copy");
        launch_tr_backward(S, prm.get(), wl.get(), w, grad.get(), stream);
        launch_tr_adam(prm.get(), adam_m.get(), adam_v.get(), grad.get(), wl.get(), lr[k], ++steps, stream);
    }
    if (loss_out && count > 0)
        cuda_check(cudaMemcpyAsync(loss_out, losses.get(), sizeof(double) * count, cudaMemcpyDeviceToHost, stream),
                   "download");
    cuda_check(cudaStreamSynchronize(stream), "trainer steps");
}

void mas_ws_trainer::evaluate(const int *idx, int count, double *rho_out)
{
    cuda_check(cudaSetDevice(device), "set device");
    for (int k = 0; k < count; ++k)
        if (idx[k] < 0 || idx[k] >= (int)samples.size())
            throw Error(ERR_INVALID, "[MAS] warm start trainer: no such sample");
    int maxn = 0;
    for (int k = 0; k < count; ++k)
        maxn = std::max(maxn, view(idx[k]).banks * 32);
    ensure_scratch(maxn);
    losses.alloc(std::max(count, 1), "warm start trainer losses");
    const WsTrainScratch w = scratch();
    for (int k = 0; k < count; ++k)
    {
        launch_tr_forward(view(idx[k]), prm.get(), wl.get(), w, stream);
        cuda_check(cudaMemcpyAsync(losses.get() + k, state_field(w.st, offsetof(WsTrainState, rho)), sizeof(double), cudaMemcpyDeviceToDevice, stream),
                   "rho copy");
    }
    if (rho_out && count > 0)
        cuda_check(cudaMemcpyAsync(rho_out, losses.get(), sizeof(double) * count, cudaMemcpyDeviceToHost, stream),
                   "download");
    cuda_check(cudaStreamSynchronize(stream), "trainer evaluate");
}

namespace
{
    template <class F>
    int tguard(mas_ws_trainer *t, F &&f)
    {
        try
        {
            f();
            if (t)
                t->last_error.clear();
            return MAS_OK;
        }
        catch (const Error &e)
        {
            if (t)
                t->last_error = e.what();
            return e.code;
        }
        catch (const std::bad_alloc &)
        {
            if (t)
                t->last_error = "[MAS] host allocation failed";
            return ERR_OOM;
        }
        catch (const std::exception &e)
        {
            if (t)
                t->last_error = std::string("[MAS] ") + e.what();
            return ERR_INVALID;
        }
    }
    std::string g_trainer_create_error;
} // namespace

extern "C" int mas_ws_trainer_create(const float *params, long long count, mas_ws_trainer **out)
{
    if (!out)
        return MAS_ERR_INVALID;
    *out = nullptr;
    auto *t = new mas_ws_trainer();
    const int rc = tguard(t, [&] { t->init(params, count); });
    if (rc != MAS_OK)
    {
        g_trainer_create_error = t->last_error;
        delete t;
        return rc;
    }
    *out = t;
    return MAS_OK;
}

extern "C" void mas_ws_trainer_destroy(mas_ws_trainer *t) { delete t; }

extern "C" int mas_ws_trainer_sample_count(const mas_ws_trainer *t) { return t ? (int)t->samples.size() : 0; }

extern "C" int mas_ws_trainer_gradient(mas_ws_trainer *t, int sample, float *grad, long long count, double *loss)
{
    if (!t || (grad && count != WS_PARAMS))
        return MAS_ERR_INVALID;
    return tguard(t, [&] { t->gradient(sample, grad, loss); });
}

extern "C" int mas_ws_trainer_train(mas_ws_trainer *t, const int *samples, const float *lr, int count,
                                    double *losses)
{
    if (!t || count < 0 || (count > 0 && (!samples || !lr)))
        return MAS_ERR_INVALID;
    return tguard(t, [&] { t->train(samples, lr, count, losses); });
}

extern "C" int mas_ws_trainer_evaluate(mas_ws_trainer *t, const int *samples, int count, double *rho)
{
    if (!t || count < 0 || (count > 0 && !samples))
        return MAS_ERR_INVALID;
    return tguard(t, [&] { t->evaluate(samples, count, rho); });
}

extern "C" int mas_ws_trainer_get_params(const mas_ws_trainer *t, float *params, long long count)
{
    if (!t || !params || count != WS_PARAMS)
        return MAS_ERR_INVALID;
    auto *tt = const_cast<mas_ws_trainer *>(t);
    return tguard(tt, [&] {
        cuda_check(cudaSetDevice(tt->device), "set device");
        cuda_check(cudaMemcpyAsync(params, tt->prm.get(), sizeof(float) * WS_PARAMS, cudaMemcpyDeviceToHost,
                                   tt->stream),
                   "download");
        cuda_check(cudaStreamSynchronize(tt->stream), "download");
    });
}

extern "C" const char *mas_ws_trainer_last_error(const mas_ws_trainer *t)
{
    return t ? t->last_error.c_str() : g_trainer_create_error.c_str();
}
