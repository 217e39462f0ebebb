// C ABI of the learned row scheduler (sdl_mlp_*, sdl_product_create_learned).
#include <memory>

#include "capi_common.h"
#include "sdl_mlp.h"

namespace sdl {
const Product *product_of(const sdl_product *P);
} // namespace sdl

using namespace sdl;

static_assert(MLP_NPARAMS == SDL_MLP_NPARAMS, "parameter count of the public header");

struct sdl_mlp
{
    Mlp net;
    explicit sdl_mlp(unsigned long long seed) : net(seed) {}
};

// sdl_product is defined in ext_api.cpp; products made here are built through it.
extern "C" sdl_status sdl_product_create(const sdl_product_desc *desc, void *stream, sdl_product **out);
namespace sdl {
sdl_product *product_new_learned(const ProductDesc &d, const Mlp &net, float margin, LearnedStats &st,
                                 cudaStream_t s);
sdl_product *product_new_learned_oneshot(const ProductDesc &d, const Mlp &net, float margin, const double *Lx,
                                         const double *dvec, const double *Ax, LearnedStats &st, cudaStream_t s);
}

extern "C" sdl_status sdl_mlp_create(unsigned long long seed, sdl_mlp **out)
{
    return guard_status("sdl_mlp_create", [&]() {
        if (!out) fail(SDL_ERR_INVALID, "NULL argument");
        *out = new sdl_mlp(seed);
    });
}

extern "C" void sdl_mlp_destroy(sdl_mlp *net) { delete net; }

extern "C" sdl_status sdl_mlp_get_params(const sdl_mlp *net, float *host)
{
    return guard_status("sdl_mlp_get_params", [&]() {
        if (!net || !host) fail(SDL_ERR_INVALID, "NULL argument");
        SDL_CUDA(cudaMemcpy(host, net->net.params.get(), MLP_NPARAMS * 4, cudaMemcpyDeviceToHost));
    });
}

extern "C" sdl_status sdl_mlp_set_params(sdl_mlp *net, const float *host)
{
    return guard_status("sdl_mlp_set_params", [&]() {
        if (!net || !host) fail(SDL_ERR_INVALID, "NULL argument");
        SDL_CUDA(cudaMemcpy(net->net.params.get(), host, MLP_NPARAMS * 4, cudaMemcpyHostToDevice));
    });
}

extern "C" sdl_status sdl_product_row_stats(const sdl_product *Ph, float *feat, float *label, void *stream)
{
    return guard_status("sdl_product_row_stats", [&]() {
        const Product *P = product_of(Ph);
        if (!P || !feat) fail(SDL_ERR_INVALID, "NULL argument");
        cudaStream_t s = pick_stream(stream);
        row_features(P->desc, P->Cp.get(), feat, label, s);
    });
}

extern "C" sdl_status sdl_mlp_gradient(const sdl_mlp *net, const float *feat, const float *label, int n,
                                       float *host_grad, float *loss)
{
    return guard_status("sdl_mlp_gradient", [&]() {
        if (!net || !feat || !label || !host_grad) fail(SDL_ERR_INVALID, "NULL argument");
        cudaStream_t s = runtime().stream;
        DevBuf<float> g(MLP_NPARAMS);
        float l = mlp_gradient(net->net, feat, label, nullptr, n, g.get(), s);
        SDL_CUDA(cudaMemcpy(host_grad, g.get(), MLP_NPARAMS * 4, cudaMemcpyDeviceToHost));
        if (loss) *loss = l;
    });
}

extern "C" sdl_status sdl_mlp_train(sdl_mlp *net, const float *feat, const float *label, long long n,
                                    int epochs, int batch, float lr, unsigned long long seed,
                                    float *final_loss)
{
    return guard_status("sdl_mlp_train", [&]() {
        if (!net || !feat || !label) fail(SDL_ERR_INVALID, "NULL argument");
        if (epochs < 0 || batch <= 0) fail(SDL_ERR_INVALID, "bad training schedule");
        float l = mlp_train(net->net, feat, label, n, epochs, batch, lr, seed, runtime().stream);
        if (final_loss) *final_loss = l;
    });
}

extern "C" sdl_status sdl_mlp_predict(const sdl_mlp *net, const float *feat, long long n, float *out,
                                      void *stream)
{
    return guard_status("sdl_mlp_predict", [&]() {
        if (!net || !feat || !out) fail(SDL_ERR_INVALID, "NULL argument");
        mlp_predict(net->net, feat, n, out, pick_stream(stream));
    });
}

extern "C" sdl_status sdl_product_create_learned(const sdl_product_desc *desc, const sdl_mlp *net,
                                                 float margin, void *stream, sdl_product **out,
                                                 sdl_learned_stats *stats)
{
    return guard_status("sdl_product_create_learned", [&]() {
        if (!desc || !net || !out) fail(SDL_ERR_INVALID, "NULL argument");
        if (!(margin >= 0.f)) fail(SDL_ERR_INVALID, "margin must be >= 0");
        *out = nullptr;
        ProductDesc d;
        d.Lp = desc->Lp;
        d.Li = desc->Li;
        d.L_map = desc->L_map;
        d.L_m = desc->L_m;
        d.L_nnz = desc->L_nnz;
        d.blocks = desc->blocks;
        d.Ap = desc->Ap;
        d.Ai = desc->Ai;
        d.A_m = desc->A_m;
        d.A_n = desc->A_n;
        d.A_nnz = desc->A_nnz;
        if (!d.Lp || !d.Ap) fail(SDL_ERR_INVALID, "NULL structure pointer");
        LearnedStats st;
        sdl_product *P = product_new_learned(d, net->net, margin, st, pick_stream(stream));
        if (stats)
        {
            stats->rows = st.rows;
            stats->term_bound = st.ub_total;
            stats->capacity = st.cap_total;
            stats->fallback_rows = st.fallback_rows;
            stats->fallback_terms = st.fallback_terms;
            stats->class_hits = st.class_hits;
            stats->scratch_bytes = product_of(P)->scratch_bytes;
        }
        *out = P;
    });
}

extern "C" sdl_status sdl_product_create_learned_filled(const sdl_product_desc *desc, const sdl_mlp *net,
                                                        float margin, const double *Lx, const double *d,
                                                        const double *Ax, void *stream, sdl_product **out,
                                                        sdl_learned_stats *stats)
{
    return guard_status("sdl_product_create_learned_filled", [&]() {
        if (!desc || !net || !out) fail(SDL_ERR_INVALID, "NULL argument");
        if (!(margin >= 0.f)) fail(SDL_ERR_INVALID, "margin must be >= 0");
        *out = nullptr;
        ProductDesc dd;
        dd.Lp = desc->Lp;
        dd.Li = desc->Li;
        dd.L_map = desc->L_map;
        dd.L_m = desc->L_m;
        dd.L_nnz = desc->L_nnz;
        dd.blocks = desc->blocks;
        dd.Ap = desc->Ap;
        dd.Ai = desc->Ai;
        dd.A_m = desc->A_m;
        dd.A_n = desc->A_n;
        dd.A_nnz = desc->A_nnz;
        if (!dd.Lp || !dd.Ap) fail(SDL_ERR_INVALID, "NULL structure pointer");
        LearnedStats st;
        sdl_product *P = product_new_learned_oneshot(dd, net->net, margin, Lx, d, Ax, st, pick_stream(stream));
        if (stats)
        {
            stats->rows = st.rows;
            stats->term_bound = st.ub_total;
            stats->capacity = st.cap_total;
            stats->fallback_rows = st.fallback_rows;
            stats->fallback_terms = st.fallback_terms;
            stats->class_hits = st.class_hits;
            stats->scratch_bytes = product_of(P)->scratch_bytes;
        }
        *out = P;
    });
}

extern "C" sdl_status sdl_product_scratch_bytes(const sdl_product *P, long long *bytes)
{
    return guard_status("sdl_product_scratch_bytes", [&]() {
        if (!P || !bytes) fail(SDL_ERR_INVALID, "NULL argument");
        *bytes = product_of(P)->scratch_bytes;
    });
}
