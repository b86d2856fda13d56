// extern "C" entry points of libp2cuda.so (declared in include/p2cuda.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "p2_solver.h"

struct p2_ctx {
    p2::Solver *s = nullptr;
    std::string err;
};

template <typename F>
static p2_status guard(p2_ctx *ctx, F &&f)
{
    if (!ctx) return P2_ERR_ARG;
    try {
        f();
        ctx->err.clear();
        return P2_OK;
    } catch (const p2::Error &e) {
        ctx->err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        ctx->err = "host allocation failed";
        return P2_ERR_NOMEM;
    } catch (...) {
        ctx->err = "unknown error";
        return P2_ERR_CUDA;
    }
}

extern "C" {

void p2_default_params(p2_params *p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // pardiso/mode.t3c:83-93
    p->p0koef = 0.3;
    p->p1koef = 1.0;
    p->p2koef = 0.0;
    p->v0koef = 1.0;
    p->v1koef = 1.0;
    p->nubeg = 1.0;
    p->nuend = 1e4;
    p->nukoef = 0.0;
    p->gxkoef = p->gykoef = 0.0;
    p->gzkoef = 0.0;
    p->pinit = 0.0;
    p->pxinit = p->pyinit = p->pzinit = 2;
    p->viscmod = 0;
    p->multinum = 2;
    for (int l = 0; l < P2_MAX_LEVELS; l++) { p->npre[l] = 4; p->npost[l] = 4; }
    p->tol = 1e-8;
    p->max_iter = 200;
    p->precision = 0;
    p->restart = 16;
    p->omega = 0.7;
    p->use_graphs = 1;
    p->smoother = 1;
}

p2_status p2_create(p2_ctx **out, int device)
{
    if (!out) return P2_ERR_ARG;
    *out = nullptr;
    p2_ctx *ctx = new (std::nothrow) p2_ctx;
    if (!ctx) return P2_ERR_NOMEM;
    p2_status st = guard(ctx, [&] {
        int n = 0;
        P2_CUDA_TRY(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) throw p2::Error(P2_ERR_ARG, "no such CUDA device");
        ctx->s = new p2::Solver(device);
    });
    if (st != P2_OK) {
        delete ctx;
        return st;
    }
    *out = ctx;
    return P2_OK;
}

void p2_destroy(p2_ctx *ctx)
{
    if (!ctx) return;
    delete ctx->s;
    delete ctx;
}

const char *p2_last_error(const p2_ctx *ctx)
{
    if (!ctx) return "null context";
    return ctx->err.c_str();
}

p2_status p2_set_grid(p2_ctx *ctx, long xnumx, long ynumy, long znumz, const double *gx, const double *gy,
                      const double *gz, int xperiodic, int yperiodic, int zperiodic, const p2_params *prm)
{
    return guard(ctx, [&] {
        if (!gx || !gy || !gz || !prm) throw p2::Error(P2_ERR_ARG, "null argument");
        if (xperiodic || yperiodic || zperiodic)
            throw p2::Error(P2_ERR_UNSUPPORTED, "periodic boundaries are not supported");
        if (prm->precision != 0 && prm->precision != 1) throw p2::Error(P2_ERR_ARG, "precision must be 0 or 1");
        if (!(prm->omega > 0 && prm->omega < 2)) throw p2::Error(P2_ERR_ARG, "omega must be in (0, 2)");
        if (prm->smoother < 0 || prm->smoother > 6 || prm->smoother == 4)
            throw p2::Error(P2_ERR_ARG, "smoother must be 0, 1, 2, 3, 5 or 6");
        if (!(prm->tol > 0)) throw p2::Error(P2_ERR_ARG, "tol must be positive");
        if (!(prm->nubeg > 0) || !(prm->nuend >= prm->nubeg)) throw p2::Error(P2_ERR_ARG, "bad nubeg/nuend");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->set_grid(xnumx, ynumy, znumz, gx, gy, gz, *prm);
    });
}

p2_status p2_set_bc(p2_ctx *ctx, const int *bondm, long bondm_len, const float *bondv1, const int *bondn1,
                    long bondnum)
{
    return guard(ctx, [&] {
        if (!bondm || !bondv1 || !bondn1 || bondnum < 0) throw p2::Error(P2_ERR_ARG, "null or negative argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->set_bc(bondm, bondm_len, bondv1, bondn1, bondnum);
    });
}

p2_status p2_set_nodes(p2_ctx *ctx, const float *nu, const float *ro, const float *nxx, const float *nxy,
                       const float *nxz, const float *nyz)
{
    return guard(ctx, [&] {
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->upload_nodes(nu, ro, nxx, nxy, nxz, nyz);
    });
}

static void finish_info(p2_solve_info *info, const p2_solve_info &r)
{
    if (info) *info = r;
}

p2_status p2_stokes_solve(p2_ctx *ctx, float *vx, float *vy, float *vz, double *pr, p2_solve_info *info)
{
    p2_solve_info r{};
    p2_status st = guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        if (!S.bc_ready) throw p2::Error(P2_ERR_STATE, "solve before p2_set_bc");
        S.set_initial(vx, vy, vz, pr);
        r = S.solve();
        S.get_solution_f32(vx, vy, vz, pr);
    });
    finish_info(info, r);
    if (st != P2_OK) return st;
    return (p2_status)r.status;
}

p2_status p2_stokes_solve_resident(p2_ctx *ctx, p2_solve_info *info)
{
    p2_solve_info r{};
    p2_status st = guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        if (!S.bc_ready) throw p2::Error(P2_ERR_STATE, "solve before p2_set_bc");
        S.set_initial(nullptr, nullptr, nullptr, nullptr);
        r = S.solve();
    });
    finish_info(info, r);
    if (st != P2_OK) return st;
    return (p2_status)r.status;
}

p2_status p2_stokes_solve_batch(p2_ctx *const *ctxs, int count, int host_threads, p2_solve_info *infos, double *ms)
{
    if (count < 0 || (count > 0 && !ctxs)) return P2_ERR_ARG;
    for (int i = 0; i < count; i++)
        if (!ctxs[i]) return P2_ERR_ARG;
    if (count == 0) {
        if (ms) *ms = 0;
        return P2_OK;
    }
    // largest instances first, so that the longest solves start at once
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const p2::Solver *sa = ctxs[a]->s, *sb = ctxs[b]->s;
        const long na = sa->L.empty() ? 0 : sa->L[0].n, nb = sb->L.empty() ? 0 : sb->L[0].n;
        return na > nb;
    });
    std::vector<p2_solve_info> res(count);
    std::vector<p2_status> sts(count, P2_OK);
    // device-side clock: events on a stream of the first context's device
    p2::Solver &S0 = *ctxs[0]->s;
    cudaStream_t clock_st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    p2_status st0 = guard(ctxs[0], [&] {
        P2_CUDA_TRY(cudaSetDevice(S0.dev));
        P2_CUDA_TRY(cudaStreamCreateWithFlags(&clock_st, cudaStreamNonBlocking));
        P2_CUDA_TRY(cudaEventCreate(&e0));
        P2_CUDA_TRY(cudaEventCreate(&e1));
        P2_CUDA_TRY(cudaEventRecord(e0, clock_st));
        P2_CUDA_TRY(cudaEventSynchronize(e0));
    });
    if (st0 == P2_OK) {
        std::atomic<int> next{0};
        auto work = [&] {
            for (int q = next++; q < count; q = next++) {
                const int i = order[q];
                sts[i] = p2_stokes_solve_resident(ctxs[i], &res[i]);
            }
        };
        int nt = host_threads > 0 ? host_threads : count;
        const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
        if (host_threads <= 0) nt = std::min(nt, hw);
        nt = std::max(1, std::min(nt, count));
        std::vector<std::thread> pool;
        try {
            for (int t = 1; t < nt; t++) pool.emplace_back(work);
        } catch (...) {
            // fewer workers than asked: the ones that started and this thread finish the batch
        }
        work();
        for (auto &t : pool) t.join();
        st0 = guard(ctxs[0], [&] {
            P2_CUDA_TRY(cudaSetDevice(S0.dev));
            P2_CUDA_TRY(cudaEventRecord(e1, clock_st));
            P2_CUDA_TRY(cudaEventSynchronize(e1));
            float t = 0;
            P2_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
            if (ms) *ms = t;
        });
    }
    cudaSetDevice(S0.dev);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (clock_st) cudaStreamDestroy(clock_st);
    if (infos)
        for (int i = 0; i < count; i++) infos[i] = res[i];
    for (int i = 0; i < count; i++)
        if (sts[i] != P2_OK) return sts[i];
    return st0;
}

p2_status p2_get_solution(p2_ctx *ctx, double *vx, double *vy, double *vz, double *pr)
{
    return guard(ctx, [&] {
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        if (!ctx->s->bc_ready) throw p2::Error(P2_ERR_STATE, "no solution");
        ctx->s->get_solution(vx, vy, vz, pr);
    });
}

p2_status p2_upload_markers(p2_ctx *ctx, long nmark, const float *markx, const float *marky, const float *markz,
                            const signed char *markt, int nrock, const double *markn0, const double *markn1,
                            const double *markro)
{
    return guard(ctx, [&] {
        if (nmark > 0 && (!markx || !marky || !markz || !markt)) throw p2::Error(P2_ERR_ARG, "null marker array");
        if (!markn0 || !markn1 || !markro) throw p2::Error(P2_ERR_ARG, "null rock table");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->upload_markers(nmark, markx, marky, markz, markt, nrock, markn0, markn1, markro);
    });
}

p2_status p2_ronurecalc_resident(p2_ctx *ctx, double *ms)
{
    return guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        P2_CUDA_TRY(cudaEventRecord(S.ev[5], S.st));
        S.ronurecalc_device();
        P2_CUDA_TRY(cudaEventRecord(S.ev[6], S.st));
        P2_CUDA_TRY(cudaEventSynchronize(S.ev[6]));
        float t = 0;
        P2_CUDA_TRY(cudaEventElapsedTime(&t, S.ev[5], S.ev[6]));
        if (ms) *ms = t;
    });
}

p2_status p2_get_nodes(p2_ctx *ctx, float *nu, float *ro, float *nxx, float *nxy, float *nxz, float *nyz)
{
    return guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        if (!S.markers_ready) throw p2::Error(P2_ERR_STATE, "no node fields computed");
        float *dst[6] = {nu, ro, nxx, nxy, nxz, nyz};
        for (int q = 0; q < 6; q++)
            if (dst[q])
                P2_CUDA_TRY(cudaMemcpyAsync(dst[q], S.mk_nodes[q], sizeof(float) * S.L[0].n, cudaMemcpyDeviceToHost,
                                            S.st));
        P2_CUDA_TRY(cudaStreamSynchronize(S.st));
    });
}

p2_status p2_ronurecalc(p2_ctx *ctx, long nmark, const float *markx, const float *marky, const float *markz,
                        const signed char *markt, int nrock, const double *markn0, const double *markn1,
                        const double *markro, float *nu, float *ro, float *nxx, float *nxy, float *nxz, float *nyz)
{
    p2_status st = p2_upload_markers(ctx, nmark, markx, marky, markz, markt, nrock, markn0, markn1, markro);
    if (st != P2_OK) return st;
    st = guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        float *src[6] = {nu, ro, nxx, nxy, nxz, nyz};
        for (int q = 0; q < 6; q++) {
            if (!src[q]) throw p2::Error(P2_ERR_ARG, "null node field");
            P2_CUDA_TRY(cudaMemcpyAsync(S.mk_nodes[q], src[q], sizeof(float) * S.L[0].n, cudaMemcpyHostToDevice,
                                        S.st));
        }
    });
    if (st != P2_OK) return st;
    st = p2_ronurecalc_resident(ctx, nullptr);
    if (st != P2_OK) return st;
    return p2_get_nodes(ctx, nu, ro, nxx, nxy, nxz, nyz);
}

p2_status p2_ronurecalc_powerlaw(p2_ctx *ctx, long nmark, const float *markx, const float *marky,
                                 const float *markz, const signed char *markt, int nrock, const double *markn0,
                                 const double *markn1, const double *markro, const double *marknu,
                                 const double *markmm, const double *val1, float *nu, float *ro, float *nxx,
                                 float *nxy, float *nxz, float *nyz)
{
    p2_status st = guard(ctx, [&] {
        if (nmark > 0 && (!markx || !marky || !markz || !markt || !val1))
            throw p2::Error(P2_ERR_ARG, "null marker array");
        if (!markn0 || !markn1 || !markro || !marknu || !markmm) throw p2::Error(P2_ERR_ARG, "null rock table");
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        S.upload_markers(nmark, markx, marky, markz, markt, nrock, markn0, markn1, markro, marknu, markmm, val1);
        float *src[6] = {nu, ro, nxx, nxy, nxz, nyz};
        for (int q = 0; q < 6; q++) {
            if (!src[q]) throw p2::Error(P2_ERR_ARG, "null node field");
            P2_CUDA_TRY(cudaMemcpyAsync(S.mk_nodes[q], src[q], sizeof(float) * S.L[0].n, cudaMemcpyHostToDevice,
                                        S.st));
        }
    });
    if (st != P2_OK) return st;
    st = p2_ronurecalc_resident(ctx, nullptr);
    if (st != P2_OK) return st;
    return p2_get_nodes(ctx, nu, ro, nxx, nxy, nxz, nyz);
}

p2_status p2_debug_apply(p2_ctx *ctx, int level, const double *x, double *y)
{
    return guard(ctx, [&] {
        if (!x || !y) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->debug_apply(level, x, y);
    });
}

p2_status p2_debug_restrict(p2_ctx *ctx, int coarse_level, const double *fine_res, double *coarse_rhs, int compat)
{
    return guard(ctx, [&] {
        if (!fine_res || !coarse_rhs) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->debug_restrict(coarse_level, fine_res, coarse_rhs, compat);
    });
}

p2_status p2_debug_prolong(p2_ctx *ctx, int coarse_level, const double *coarse_x, double *fine_x)
{
    return guard(ctx, [&] {
        if (!coarse_x || !fine_x) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->debug_prolong(coarse_level, coarse_x, fine_x);
    });
}

p2_status p2_movemark(p2_ctx *ctx, double timestep, int markmod, int outgrid, const float *vx, const float *vy, const float *vz,
                      long nmark, float *markx, float *marky, float *markz, const signed char *markt)
{
    return guard(ctx, [&] {
        if (!vx || !vy || !vz || (nmark > 0 && (!markx || !marky || !markz || !markt)))
            throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->movemark_host(timestep, markmod, outgrid, vx, vy, vz, nmark, markx, marky, markz, markt);
    });
}

p2_status p2_movemark_strain(p2_ctx *ctx, double timestep, int markmod, int outgrid, const float *vx,
                             const float *vy, const float *vz, const float *exx, const float *eyy, const float *ezz,
                             const float *exy, const float *exz, const float *eyz, long nmark, float *markx,
                             float *marky, float *markz, const signed char *markt, double *val1, float *marke)
{
    return guard(ctx, [&] {
        if (!vx || !vy || !vz || !exx || !eyy || !ezz || !exy || !exz || !eyz)
            throw p2::Error(P2_ERR_ARG, "null field");
        if (nmark > 0 && (!markx || !marky || !markz || !markt || !val1 || !marke))
            throw p2::Error(P2_ERR_ARG, "null marker array");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        const float *const e[6] = {exx, eyy, ezz, exy, exz, eyz};
        ctx->s->movemark_strain_host(timestep, markmod, outgrid, vx, vy, vz, e, nmark, markx, marky, markz, markt,
                                     val1, marke);
    });
}

p2_status p2_movemark_resident(p2_ctx *ctx, double timestep, int markmod, int outgrid, double *ms)
{
    return guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        P2_CUDA_TRY(cudaEventRecord(S.ev[5], S.st));
        S.movemark_device(timestep, markmod, outgrid);
        P2_CUDA_TRY(cudaEventRecord(S.ev[6], S.st));
        P2_CUDA_TRY(cudaEventSynchronize(S.ev[6]));
        float t = 0;
        P2_CUDA_TRY(cudaEventElapsedTime(&t, S.ev[5], S.ev[6]));
        if (ms) *ms = t;
    });
}

p2_status p2_get_markers(p2_ctx *ctx, float *markx, float *marky, float *markz)
{
    return guard(ctx, [&] {
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->get_markers(markx, marky, markz);
    });
}

p2_status p2_stress_strain(p2_ctx *ctx, float *sxx, float *syy, float *szz, float *sxy, float *sxz, float *syz,
                           float *exx, float *eyy, float *ezz, float *exy, float *exz, float *eyz, double vrange[6])
{
    return guard(ctx, [&] {
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        float *const s[6] = {sxx, syy, szz, sxy, sxz, syz};
        float *const e[6] = {exx, eyy, ezz, exy, exz, eyz};
        ctx->s->stress_strain(s, e, vrange);
    });
}

p2_status p2_effbulk_visc(p2_ctx *ctx, const float *ro, const float *nxx, const float *nxy, const float *nxz,
                          const float *nyz, const float *exx, const float *eyy, const float *ezz, const float *exy,
                          const float *exz, const float *eyz, const float *sxx, const float *syy, const float *szz,
                          const float *sxy, const float *sxz, const float *syz, p2_effbulk *out)
{
    return guard(ctx, [&] {
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        const float *const e[6] = {exx, eyy, ezz, exy, exz, eyz};
        const float *const s[6] = {sxx, syy, szz, sxy, sxz, syz};
        ctx->s->effbulk(ro, nxx, nxy, nxz, nyz, e, s, out);
    });
}

void p2_default_heat_params(p2_heat_params *hp)
{
    if (!hp) return;
    std::memset(hp, 0, sizeof(*hp));
    // pardiso/mode.t3c:100-110 (T_ITERATIONS_PARAMETERS), 118-121, and the
    // maxtkstep column of the SAVEFL lines (mode.t3c:9-13)
    hp->heatmin = 1e-4;
    hp->multinumt = 0;
    hp->multicyct = 1;
    hp->multittt[0][0] = 10;
    hp->multittt[1][0] = 0;
    hp->t0koef = 1.0;
    hp->t1koef = 1.0;
    hp->heatdif = 1.0;
    hp->frictyn = 1;
    hp->adiabyn = 1;
    hp->tdeep = 3055;
    hp->zdeep = 3800;
    hp->maxtkstep = 25.0;
    hp->max_cycles = 10000;
}

p2_status p2_heat_set_bc(p2_ctx *ctx, const int *bondm, long bondm_len, const float *bondv1, const int *bondn1,
                         long bondnum)
{
    return guard(ctx, [&] {
        if (!bondm || !bondv1 || !bondn1 || bondnum < 0) throw p2::Error(P2_ERR_ARG, "bad boundary tables");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->heat_set_bc(bondm, bondm_len, bondv1, bondn1, bondnum);
    });
}

p2_status p2_titerate(p2_ctx *ctx, const p2_heat_params *hp, double timestep, float *tk, const float *kt,
                      const float *cp, const float *ro, const float *ht, const float *et, const float *vx,
                      const float *vy, const float *vz, const double *pr, const float *const *stress_strain,
                      long marknum, const float *markx, const float *marky, const float *markz,
                      const signed char *markt, float *markk, p2_heat_info *info)
{
    return guard(ctx, [&] {
        if (!hp) throw p2::Error(P2_ERR_ARG, "null parameters");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        p2_heat_info r = ctx->s->titerate(*hp, timestep, tk, kt, cp, ro, ht, et, vx, vy, vz, pr, stress_strain,
                                          marknum, markx, marky, markz, markt, markk);
        if (info) *info = r;
    });
}

p2_status p2_autotune(p2_ctx *ctx, int trial_iters, p2_tune_info *info)
{
    return guard(ctx, [&] {
        p2::Solver &S = *ctx->s;
        P2_CUDA_TRY(cudaSetDevice(S.dev));
        p2_tune_info r = S.autotune(trial_iters);
        if (info) *info = r;
    });
}

p2_status p2_debug_time_smoother(p2_ctx *ctx, int level, int passes, double *ms_per_pass)
{
    return guard(ctx, [&] {
        if (!ms_per_pass) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        *ms_per_pass = ctx->s->debug_time_smoother(level, passes);
    });
}

p2_status p2_debug_smooth(p2_ctx *ctx, int level, int sweeps, const double *b, double *x)
{
    return guard(ctx, [&] {
        if (!b || !x) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->debug_smooth(level, sweeps, b, x);
    });
}

p2_status p2_debug_time_sweep(p2_ctx *ctx, int level, int sweeps, double *ms_per_sweep)
{
    return guard(ctx, [&] {
        if (!ms_per_sweep) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        *ms_per_sweep = ctx->s->debug_time_sweep(level, sweeps);
    });
}

p2_status p2_debug_rows_kernel(p2_ctx *ctx, int variant)
{
    return guard(ctx, [&] {
        if (variant < 0 || variant > 2) throw p2::Error(P2_ERR_ARG, "rows kernel variant must be 0..2");
        ctx->s->dbg_rows_variant = variant;
        ctx->s->drop_graphs_public();
    });
}

p2_status p2_debug_vcycle(p2_ctx *ctx, const double *b, double *x)
{
    return guard(ctx, [&] {
        if (!b || !x) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->debug_vcycle(b, x);
    });
}

p2_status p2_debug_time_stage(p2_ctx *ctx, int stage, int level, int variant, int reps, double *ms)
{
    return guard(ctx, [&] {
        if (!ms) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        *ms = ctx->s->debug_time_stage(stage, level, variant, reps);
    });
}

p2_status p2_debug_level_fields(p2_ctx *ctx, float *nu, float *ro)
{
    return guard(ctx, [&] {
        if (!nu || !ro) throw p2::Error(P2_ERR_ARG, "null argument");
        P2_CUDA_TRY(cudaSetDevice(ctx->s->dev));
        ctx->s->debug_level_fields(nu, ro);
    });
}

}  // extern "C"
