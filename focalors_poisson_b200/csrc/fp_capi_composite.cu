// C ABI (include/fp_capi.h): composite-geometry solver.
#include "../../include/fp_capi.h"
#include "fp_batch.h"
#include "fp_composite.h"

#include <set>

using namespace fpb;

namespace fpb
{
// Device side of fp_composite_solve_async: two slots, each a landing area for one call's right-hand sides and
// ghosts (written by host-to-device copies on `in`) and an outbox for its solution (read by device-to-host
// copies on `out`); the solve itself runs in the solver's own work fields on the caller's stream.
struct Pipeline
{
    cudaStream_t        in = nullptr, out = nullptr;
    std::vector<DevBuf> land[2], land_ghost[2], outbox[2];
    cudaEvent_t         landed[2] = {}, land_free[2] = {}, solved[2] = {}, out_done[2] = {};
    int                 next = 0, last = -1;  // slot of the next call, slot of the last queued one
    long long           pending = 0;          // calls queued since the last wait
    std::set<const void*> out_ptrs;           // host outputs of the pending calls
    // outcome bookkeeping of the last call
    BatchBase*          refined = nullptr;    // batch whose deferred refinement it queued, if any
    int                 form = 0, max_refine = 0, steps = 0;
    double              rel_tol = 0, change = 0;
    GmresInfo           gi;

    Pipeline()
    {
        FPB_CUDA(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking));
        FPB_CUDA(cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking));
        for (int q = 0; q < 2; ++q)
            for (cudaEvent_t* e : {&landed[q], &land_free[q], &solved[q], &out_done[q]})
                FPB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    ~Pipeline()
    {
        cudaStreamSynchronize(in);
        cudaStreamSynchronize(out);
        for (int q = 0; q < 2; ++q)
            for (cudaEvent_t e : {landed[q], land_free[q], solved[q], out_done[q]})
                if (e) cudaEventDestroy(e);
        cudaStreamDestroy(in);
        cudaStreamDestroy(out);
    }
};
}  // namespace fpb

struct fp_composite
{
    std::unique_ptr<Composite> c;
    std::vector<DevBuf>        fields, ghosts;
    // Spectral direct path (fp_batch.h) for geometries it covers: a batch of this one problem in FP64
    // (solves) and, built on first use, in FP32 (inner solves of refinement).
    BatchProblemDesc           desc;
    std::unique_ptr<BatchBase> sp64, sp32;
    std::unique_ptr<Pipeline>  pipe;  // fp_composite_solve_async, created on first use
};

namespace
{
std::unique_ptr<Composite> make_composite(const fp_geometry* g, int m, double tol, int max_iter, int flags,
                                          const std::vector<std::array<int, 2>>& ext = {})
{
    if (!g || g->n_domains <= 0 || !g->nx || !g->ny || !g->hx || !g->hy || !g->bc)
        throw Error(FP_ERR_INVALID, "incomplete geometry description");
    if (g->n_connections > 0 && !g->connections) throw Error(FP_ERR_INVALID, "null connection list");
    std::vector<Domain> doms(g->n_domains);
    for (int d = 0; d < g->n_domains; ++d)
    {
        doms[d].nx = g->nx[d];
        doms[d].ny = g->ny[d];
        doms[d].hx = g->hx[d];
        doms[d].hy = g->hy[d];
        for (int f = 0; f < 4; ++f) doms[d].bc[f] = g->bc[4 * d + f];
    }
    std::vector<std::array<int, 3>> conns(g->n_connections);
    for (int k = 0; k < g->n_connections; ++k)
        conns[k] = {g->connections[3 * k], g->connections[3 * k + 1], g->connections[3 * k + 2]};
    const int mode = (flags & FP_GMRES_FULLFIELD) ? GMRES_FULLFIELD : GMRES_INTERFACE;
    return std::unique_ptr<Composite>(
        new Composite(doms, conns, g->root, m, tol, max_iter, mode, (flags & FP_NO_INTERFACE_INVERSE) == 0, ext));
}
}  // namespace

namespace
{
// Every other entry point first lets the queued pipelined solves finish: they share the solver's work
// fields and scratch, possibly on another stream.
void drain(fp_composite* c)
{
    if (c && c->pipe && c->pipe->pending) FPB_CUDA(cudaStreamSynchronize(c->pipe->out));
}

// One solve of the given FP_FORM_* on device fields. Returns the batch whose refinement was queued without
// waiting (defer, spectral refinement forms), else nullptr.
BatchBase* solve_form(fp_composite* c, double* const* f, const double* const* g, int form, double rel_tol,
                      int max_refine, cudaStream_t s, bool defer, int* steps, double* change, GmresInfo* gi)
{
    *steps  = 0;
    *change = 0;
    if (form == FP_FORM_F64)
    {
        if (c->sp64) c->sp64->solve(f, g, 0, s);
        else c->c->solve(f, g, s, gi);
        return nullptr;
    }
    const bool f32 = form != FP_FORM_F64IR;
    if (!c->sp64)
    {
        *steps = c->c->solve_ir(f, g, s, rel_tol, max_refine, change, gi, f32);
        return nullptr;
    }
    if (f32 && !c->sp32)
    {
        c->sp32 = make_batch({c->desc}, 1);
        c->sp32->autotune(s);
    }
    BatchBase* first = form == FP_FORM_MIXEDIR ? c->sp64.get() : nullptr;
    BatchBase* b     = f32 ? c->sp32.get() : c->sp64.get();
    *steps           = b->refine(f, g, rel_tol, max_refine, s, change, first, defer);
    return *steps < 0 ? b : nullptr;
}

// Stages host or device fields, runs `body` on device pointers, copies results back for host calls.
template <typename F>
void with_device_fields(fp_composite* c, double* const* fields, const double* const* ghosts, int flags,
                        cudaStream_t s, F&& body)
{
    if (!c) throw Error(FP_ERR_INVALID, "null solver");
    drain(c);
    if (!fields) throw Error(FP_ERR_INVALID, "null field list");
    const auto& doms = c->c->domains();
    const int   nd   = (int)doms.size();
    for (int d = 0; d < nd; ++d)
        if (!fields[d]) throw Error(FP_ERR_INVALID, "null field pointer");
    if (flags & FP_DEVICE)
    {
        body(fields, ghosts);
        if (flags & FP_SYNC) FPB_CUDA(cudaStreamSynchronize(s));
        return;
    }
    c->fields.resize(nd);
    c->ghosts.resize(4 * nd);
    std::vector<double*>       dev(nd);
    std::vector<const double*> gdev(4 * nd, nullptr);
    for (int d = 0; d < nd; ++d)
    {
        const size_t bytes = doms[d].cells() * sizeof(double);
        c->fields[d].ensure(bytes);
        dev[d] = c->fields[d].as<double>();
        FPB_CUDA(cudaMemcpyAsync(dev[d], fields[d], bytes, cudaMemcpyHostToDevice, s));
        for (int f = 0; f < 4 && ghosts; ++f)
        {
            if (!ghosts[4 * d + f]) continue;
            const size_t gb = (size_t)(f < 2 ? doms[d].ny : doms[d].nx) * sizeof(double);
            c->ghosts[4 * d + f].ensure(gb);
            FPB_CUDA(cudaMemcpyAsync(c->ghosts[4 * d + f].get(), ghosts[4 * d + f], gb, cudaMemcpyHostToDevice, s));
            gdev[4 * d + f] = c->ghosts[4 * d + f].as<double>();
        }
    }
    body(dev.data(), gdev.data());
    for (int d = 0; d < nd; ++d)
        FPB_CUDA(cudaMemcpyAsync(fields[d], dev[d], doms[d].cells() * sizeof(double), cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
}

void fill_info(fp_solve_info* info, const GmresInfo& gi, int refinements, double change)
{
    if (!info) return;
    info->gmres_iterations = gi.iterations;
    info->gmres_restarts   = gi.restarts;
    info->gmres_residual   = gi.residual;
    info->converged        = gi.converged ? 1 : 0;
    info->refinements      = refinements;
    info->rel_change       = change;
}
}  // namespace

extern "C" {

int fp_composite_create(const fp_geometry* g, int m, double tol, int max_iter, int flags, fp_composite** out)
{
    return guarded([&] {
        if (!out) throw Error(FP_ERR_INVALID, "null output handle");
        *out = nullptr;
        require_device();
        std::unique_ptr<fp_composite> h(new fp_composite());
        h->c = make_composite(g, m, tol, max_iter, flags);
        if (!(flags & (FP_GMRES_FULLFIELD | FP_NO_SPECTRAL)))
        {
            for (int d = 0; d < g->n_domains; ++d)
            {
                Domain D;
                D.nx = g->nx[d];
                D.ny = g->ny[d];
                D.hx = g->hx[d];
                D.hy = g->hy[d];
                for (int f = 0; f < 4; ++f) D.bc[f] = g->bc[4 * d + f];
                h->desc.doms.push_back(D);
            }
            for (int k = 0; k < g->n_connections; ++k)
            {
                const int a = g->connections[3 * k], f = g->connections[3 * k + 1], b = g->connections[3 * k + 2];
                h->desc.conns.push_back({a, f, b});
                h->desc.doms[a].bc[f]     = BC_ADJACENTED;
                h->desc.doms[b].bc[f ^ 1] = BC_ADJACENTED;
            }
            try
            {
                h->sp64 = make_batch({h->desc}, 0);
                h->sp64->autotune(0);
                FPB_CUDA(cudaDeviceSynchronize());
            }
            catch (const Error& e)
            {
                if (e.code != FP_ERR_UNSUPPORTED) throw;
                h->sp64.reset();  // outside the spectral path's scope: Schur GMRES
            }
        }
        // the Schur GMRES path builds its matrices and interface inverses here, so that no solve pays for them
        if (!h->sp64)
        {
            h->c->prepare();
            FPB_CUDA(cudaDeviceSynchronize());
        }
        *out = h.release();
    });
}

int fp_composite_set_parameter(fp_composite* c, int m, double tol, int max_iter)
{
    return guarded([&] {
        if (!c) throw Error(FP_ERR_INVALID, "null solver");
        c->c->set_parameter(m, tol, max_iter);
    });
}

int fp_composite_solve_f64(fp_composite* c, double* const* fields, const double* const* ghosts, int flags,
                           void* stream, fp_solve_info* info)
{
    GmresInfo gi;
    int       rc = guarded([&] {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        with_device_fields(c, fields, ghosts, flags, s, [&](double* const* f, const double* const* g) {
            if (c->sp64) c->sp64->solve(f, g, 0, s);  // exact interface solve: nothing to converge
            else c->c->solve(f, g, s, &gi);
        });
        if ((flags & FP_CHECK_CONVERGENCE) && !gi.converged)
            throw Error(FP_ERR_NOT_CONVERGED, "GMRES stopped at max_iter above tol (residual " +
                                                  std::to_string(gi.residual) + ")");
    });
    fill_info(info, gi, 0, 0.0);
    return rc;
}

int fp_composite_solve_f32ir(fp_composite* c, double* const* fields, const double* const* ghosts, int flags,
                             void* stream, double rel_tol, int max_refine, fp_solve_info* info)
{
    GmresInfo gi;
    int       steps  = 0;
    double    change = 0;
    int       rc     = guarded([&] {
        if (!(rel_tol > 0) || max_refine < 1) throw Error(FP_ERR_INVALID, "rel_tol must be > 0 and max_refine >= 1");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        with_device_fields(c, fields, ghosts, flags, s, [&](double* const* f, const double* const* g) {
            const bool f32 = (flags & FP_IR_INNER_F64) == 0;
            if (c->sp64)
            {
                if (f32 && !c->sp32)
                {
                    c->sp32 = make_batch({c->desc}, 1);
                    c->sp32->autotune(s);
                }
                BatchBase* first = (f32 && (flags & FP_IR_FIRST_F64)) ? c->sp64.get() : nullptr;
                steps = (f32 ? c->sp32 : c->sp64)->refine(f, g, rel_tol, max_refine, s, &change, first);
            }
            else
                steps = c->c->solve_ir(f, g, s, rel_tol, max_refine, &change, &gi, f32);
        });
        if ((flags & FP_CHECK_CONVERGENCE) && steps >= max_refine && !(change <= rel_tol))
            throw Error(FP_ERR_NOT_CONVERGED, "iterative refinement stopped at max_refine (relative change " +
                                                  std::to_string(change) + ")");
    });
    fill_info(info, gi, steps, change);
    return rc;
}

int fp_composite_adjoint_f64(fp_composite* c, double* const* fields, int flags, void* stream, fp_solve_info* info)
{
    GmresInfo gi;
    int       rc = guarded([&] {
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        with_device_fields(c, fields, nullptr, flags, s, [&](double* const* f, const double* const*) {
            if (c->sp64)  // H A^-1 g = H * (spectral solve of H^-1 g, which scales by H again)
            {
                c->c->require_nonsingular();
                c->c->scale_fields(f, false, s);
                c->sp64->solve(f, nullptr, 0, s);
                c->c->scale_fields(f, true, s);
            }
            else
                c->c->solve_adjoint(f, s, &gi);
        });
        if ((flags & FP_CHECK_CONVERGENCE) && !gi.converged)
            throw Error(FP_ERR_NOT_CONVERGED, "GMRES stopped at max_iter above tol (residual " +
                                                  std::to_string(gi.residual) + ")");
    });
    fill_info(info, gi, 0, 0.0);
    return rc;
}

int fp_composite_adjoint_f32ir(fp_composite* c, double* const* fields, int flags, void* stream, double rel_tol,
                               int max_refine, fp_solve_info* info)
{
    GmresInfo gi;
    int       steps  = 0;
    double    change = 0;
    int       rc     = guarded([&] {
        if (!(rel_tol > 0) || max_refine < 1) throw Error(FP_ERR_INVALID, "rel_tol must be > 0 and max_refine >= 1");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        with_device_fields(c, fields, nullptr, flags, s, [&](double* const* f, const double* const*) {
            const bool f32 = (flags & FP_IR_INNER_F64) == 0;
            if (c->sp64)
            {
                c->c->require_nonsingular();
                if (f32 && !c->sp32)
                {
                    c->sp32 = make_batch({c->desc}, 1);
                    c->sp32->autotune(s);
                }
                c->c->scale_fields(f, false, s);
                steps = (f32 ? c->sp32 : c->sp64)->refine(f, nullptr, rel_tol, max_refine, s, &change);
                c->c->scale_fields(f, true, s);
            }
            else
                steps = c->c->solve_adjoint_ir(f, s, rel_tol, max_refine, &change, &gi, f32);
        });
        if ((flags & FP_CHECK_CONVERGENCE) && steps >= max_refine && !(change <= rel_tol))
            throw Error(FP_ERR_NOT_CONVERGED, "iterative refinement stopped at max_refine (relative change " +
                                                  std::to_string(change) + ")");
    });
    fill_info(info, gi, steps, change);
    return rc;
}

int fp_composite_solve_async(fp_composite* c, const double* const* rhs, double* const* out,
                             const double* const* ghosts, int form, double rel_tol, int max_refine, void* stream)
{
    return guarded([&] {
        if (!c) throw Error(FP_ERR_INVALID, "null solver");
        if (!rhs || !out) throw Error(FP_ERR_INVALID, "null field list");
        if (form < FP_FORM_F64 || form > FP_FORM_MIXEDIR) throw Error(FP_ERR_INVALID, "form must be one of FP_FORM_*");
        if (form != FP_FORM_F64 && (!(rel_tol > 0) || max_refine < 1))
            throw Error(FP_ERR_INVALID, "rel_tol must be > 0 and max_refine >= 1");
        const auto& doms = c->c->domains();
        const int   nd   = (int)doms.size();
        for (int d = 0; d < nd; ++d)
            if (!rhs[d] || !out[d]) throw Error(FP_ERR_INVALID, "null field pointer");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (!c->pipe) c->pipe.reset(new Pipeline());
        Pipeline& P = *c->pipe;
        const int q = P.next;
        c->fields.resize(nd);
        c->ghosts.resize(4 * nd);
        P.land[q].resize(nd);
        P.outbox[q].resize(nd);
        P.land_ghost[q].resize(4 * nd);
        // slot q's landing area is free once the copy out of it by the call two back has run; an input that is
        // the output of a queued call waits for the copies out (in order on one stream)
        FPB_CUDA(cudaStreamWaitEvent(P.in, P.land_free[q], 0));
        bool alias = false;
        for (int d = 0; d < nd; ++d)
        {
            alias = alias || P.out_ptrs.count(rhs[d]);
            for (int f = 0; f < 4 && ghosts; ++f) alias = alias || (ghosts[4 * d + f] && P.out_ptrs.count(ghosts[4 * d + f]));
        }
        if (alias && P.last >= 0) FPB_CUDA(cudaStreamWaitEvent(P.in, P.out_done[P.last], 0));
        std::vector<double*>       work(nd);
        std::vector<const double*> gwork(4 * nd, nullptr);
        for (int d = 0; d < nd; ++d)
        {
            const size_t bytes = doms[d].cells() * sizeof(double);
            c->fields[d].ensure(bytes);
            P.land[q][d].ensure(bytes);
            P.outbox[q][d].ensure(bytes);
            work[d] = c->fields[d].as<double>();
            FPB_CUDA(cudaMemcpyAsync(P.land[q][d].get(), rhs[d], bytes, cudaMemcpyHostToDevice, P.in));
            for (int f = 0; f < 4 && ghosts; ++f)
            {
                if (!ghosts[4 * d + f]) continue;
                const size_t gb = (size_t)(f < 2 ? doms[d].ny : doms[d].nx) * sizeof(double);
                P.land_ghost[q][4 * d + f].ensure(gb);
                c->ghosts[4 * d + f].ensure(gb);
                FPB_CUDA(cudaMemcpyAsync(P.land_ghost[q][4 * d + f].get(), ghosts[4 * d + f], gb,
                                         cudaMemcpyHostToDevice, P.in));
                gwork[4 * d + f] = c->ghosts[4 * d + f].as<double>();
            }
        }
        FPB_CUDA(cudaEventRecord(P.landed[q], P.in));
        FPB_CUDA(cudaStreamWaitEvent(s, P.landed[q], 0));
        for (int d = 0; d < nd; ++d)
        {
            FPB_CUDA(cudaMemcpyAsync(work[d], P.land[q][d].get(), doms[d].cells() * sizeof(double),
                                     cudaMemcpyDeviceToDevice, s));
            for (int f = 0; f < 4; ++f)
                if (gwork[4 * d + f])
                    FPB_CUDA(cudaMemcpyAsync(const_cast<double*>(gwork[4 * d + f]), P.land_ghost[q][4 * d + f].get(),
                                             P.land_ghost[q][4 * d + f].bytes(), cudaMemcpyDeviceToDevice, s));
        }
        FPB_CUDA(cudaEventRecord(P.land_free[q], s));
        int        steps  = 0;
        double     change = 0;
        GmresInfo  gi;
        BatchBase* refined = solve_form(c, work.data(), ghosts ? gwork.data() : nullptr, form, rel_tol, max_refine,
                                        s, true, &steps, &change, &gi);
        FPB_CUDA(cudaStreamWaitEvent(s, P.out_done[q], 0));  // slot q's outbox read out by the call two back
        for (int d = 0; d < nd; ++d)
            FPB_CUDA(cudaMemcpyAsync(P.outbox[q][d].get(), work[d], doms[d].cells() * sizeof(double),
                                     cudaMemcpyDeviceToDevice, s));
        FPB_CUDA(cudaEventRecord(P.solved[q], s));
        FPB_CUDA(cudaStreamWaitEvent(P.out, P.solved[q], 0));
        for (int d = 0; d < nd; ++d)
            FPB_CUDA(cudaMemcpyAsync(out[d], P.outbox[q][d].get(), doms[d].cells() * sizeof(double),
                                     cudaMemcpyDeviceToHost, P.out));
        FPB_CUDA(cudaEventRecord(P.out_done[q], P.out));
        for (int d = 0; d < nd; ++d) P.out_ptrs.insert(out[d]);
        P.last       = q;
        P.next       = q ^ 1;
        P.pending   += 1;
        P.form       = form;
        P.rel_tol    = rel_tol;
        P.max_refine = max_refine;
        P.steps      = steps;
        P.change     = change;
        P.gi         = gi;
        if (refined) P.refined = refined;
    });
}

int fp_composite_wait(fp_composite* c, int flags, fp_solve_info* info)
{
    GmresInfo gi;
    int       steps  = 0;
    double    change = 0;
    int       rc     = guarded([&] {
        if (!c) throw Error(FP_ERR_INVALID, "null solver");
        if (!c->pipe || c->pipe->pending == 0) return;
        Pipeline& P = *c->pipe;
        FPB_CUDA(cudaStreamSynchronize(P.out));
        P.pending = 0;
        P.out_ptrs.clear();
        gi     = P.gi;
        steps  = P.steps;
        change = P.change;
        if (P.refined)
        {
            BatchBase* b = P.refined;
            P.refined    = nullptr;
            b->refine_result(&steps, &change);
        }
        if (flags & FP_CHECK_CONVERGENCE)
        {
            if (!gi.converged)
                throw Error(FP_ERR_NOT_CONVERGED, "GMRES stopped at max_iter above tol (residual " +
                                                      std::to_string(gi.residual) + ")");
            if (P.form != FP_FORM_F64 && steps >= P.max_refine && !(change <= P.rel_tol))
                throw Error(FP_ERR_NOT_CONVERGED, "iterative refinement stopped at max_refine (relative change " +
                                                      std::to_string(change) + ")");
        }
    });
    fill_info(info, gi, steps, change);
    return rc;
}

int fp_composite_part_create(const fp_geometry* g, int m, double tol, int max_iter, int flags, int n_ext,
                             const int* ext_faces, fp_composite** out)
{
    return guarded([&] {
        if (!out) throw Error(FP_ERR_INVALID, "null output handle");
        *out = nullptr;
        if (n_ext < 0 || (n_ext > 0 && !ext_faces)) throw Error(FP_ERR_INVALID, "bad external child list");
        if (!g || g->n_domains <= 0 || !g->nx || !g->ny) throw Error(FP_ERR_INVALID, "incomplete geometry description");
        require_device();
        const int r = g->root >= 0 ? g->root : 0;
        if (n_ext > 0 && (g->root < 0 || r >= g->n_domains))
            throw Error(FP_ERR_INVALID, "a root part names its root domain");
        std::vector<std::array<int, 2>> ext;
        for (int k = 0; k < n_ext; ++k)
        {
            const int f = ext_faces[k];
            if (f < 0 || f > 3) throw Error(FP_ERR_INVALID, "external child face out of range");
            ext.push_back({f, f < 2 ? g->ny[r] : g->nx[r]});
        }
        std::unique_ptr<fp_composite> h(new fp_composite());
        h->c = make_composite(g, m, tol, max_iter, flags & ~FP_GMRES_FULLFIELD, ext);
        if (n_ext == 0)
        {
            h->c->prepare();
            FPB_CUDA(cudaDeviceSynchronize());
        }
        *out = h.release();
    });
}

int fp_composite_part_schur(fp_composite* c, int face, double* S, void* stream)
{
    return guarded([&] {
        if (!c || !S) throw Error(FP_ERR_INVALID, "null argument");
        c->c->part_schur(face, S, static_cast<cudaStream_t>(stream));
    });
}

int fp_composite_set_external_schur(fp_composite* c, int k, const double* S)
{
    return guarded([&] {
        if (!c || !S) throw Error(FP_ERR_INVALID, "null argument");
        c->c->set_external_schur(k, S);
    });
}

namespace
{
void fill_part_info(fp_solve_info* info, const GmresInfo& gi)
{
    if (!info) return;
    info->gmres_iterations = gi.iterations;
    info->gmres_restarts   = gi.restarts;
    info->gmres_residual   = gi.residual;
    info->converged        = gi.converged ? 1 : 0;
    info->refinements      = 0;
    info->rel_change       = 0.0;
}
void check_fields(fp_composite* c, double* const* fields)
{
    if (!c) throw Error(FP_ERR_INVALID, "null solver");
    if (!fields) throw Error(FP_ERR_INVALID, "null field list");
    for (size_t d = 0; d < c->c->domains().size(); ++d)
        if (!fields[d]) throw Error(FP_ERR_INVALID, "null field pointer");
}
}  // namespace

int fp_composite_part_upward(fp_composite* c, double* const* fields, const double* const* ghosts, int face,
                             double* edge_out, void* stream, fp_solve_info* info)
{
    GmresInfo gi;
    const int rc = guarded([&] {
        check_fields(c, fields);
        if (!edge_out) throw Error(FP_ERR_INVALID, "null edge buffer");
        c->c->part_upward(fields, ghosts, face, edge_out, static_cast<cudaStream_t>(stream), &gi);
    });
    fill_part_info(info, gi);
    return rc;
}

int fp_composite_part_downward(fp_composite* c, double* const* fields, int face, const double* parent_edge,
                               void* stream, fp_solve_info* info)
{
    GmresInfo gi;
    const int rc = guarded([&] {
        check_fields(c, fields);
        if (!parent_edge) throw Error(FP_ERR_INVALID, "null edge buffer");
        c->c->part_downward(fields, face, parent_edge, static_cast<cudaStream_t>(stream), &gi);
    });
    fill_part_info(info, gi);
    return rc;
}

int fp_composite_root_solve(fp_composite* c, double* const* fields, const double* const* ghosts,
                            const double* const* child_edges, double* const* edges_out, void* stream,
                            fp_solve_info* info)
{
    GmresInfo gi;
    const int rc = guarded([&] {
        check_fields(c, fields);
        const int n = c->c->external_children();
        for (int k = 0; k < n; ++k)
            if (!child_edges || !child_edges[k] || !edges_out || !edges_out[k])
                throw Error(FP_ERR_INVALID, "null edge buffer");
        c->c->root_solve(fields, ghosts, child_edges, edges_out, static_cast<cudaStream_t>(stream), &gi);
    });
    fill_part_info(info, gi);
    return rc;
}

int fp_composite_residual(fp_composite* c, const double* const* u, const double* const* rhs,
                          const double* const* ghosts, void* stream, double* rel_residual)
{
    return guarded([&] {
        if (!c || !u || !rhs || !rel_residual) throw Error(FP_ERR_INVALID, "null argument");
        drain(c);
        *rel_residual = c->c->residual_norm(u, rhs, ghosts, static_cast<cudaStream_t>(stream));
    });
}

int fp_composite_tree(const fp_composite* c, int* root, int* level_of)
{
    return guarded([&] {
        if (!c || !root || !level_of) throw Error(FP_ERR_INVALID, "null argument");
        const Tree& t = c->c->tree();
        *root         = t.root;
        for (size_t l = 0; l < t.levels.size(); ++l)
            for (int d : t.levels[l]) level_of[d] = (int)l;
    });
}

int fp_composite_destroy(fp_composite* c)
{
    return guarded([&] { delete c; });
}

}  // extern "C"
