// C ABI (include/fp_capi.h): batched composite solves.
#include "../../include/fp_capi.h"
#include "fp_batch.h"

using namespace fpb;

struct fp_batch
{
    std::unique_ptr<BatchBase> b;
};

extern "C" {

int fp_batch_create(const fp_geometry* problems, int n_problems, int flags, fp_batch** out)
{
    return guarded([&] {
        if (!out) throw Error(FP_ERR_INVALID, "null output handle");
        *out = nullptr;
        if (!problems || n_problems <= 0) throw Error(FP_ERR_INVALID, "empty problem list");
        require_device();
        std::vector<BatchProblemDesc> probs(n_problems);
        for (int p = 0; p < n_problems; ++p)
        {
            const fp_geometry* g = problems + p;
            if (!g->nx || !g->ny || !g->hx || !g->hy || !g->bc || g->n_domains <= 0)
                throw Error(FP_ERR_INVALID, "incomplete geometry description of problem " + std::to_string(p));
            if (g->n_connections > 0 && !g->connections) throw Error(FP_ERR_INVALID, "null connection list");
            auto& P = probs[p];
            P.doms.resize(g->n_domains);
            for (int d = 0; d < g->n_domains; ++d)
            {
                P.doms[d].nx = g->nx[d];
                P.doms[d].ny = g->ny[d];
                P.doms[d].hx = g->hx[d];
                P.doms[d].hy = g->hy[d];
                for (int f = 0; f < 4; ++f) P.doms[d].bc[f] = g->bc[4 * d + f];
            }
            for (int k = 0; k < g->n_connections; ++k)
            {
                const int a = g->connections[3 * k], f = g->connections[3 * k + 1], b = g->connections[3 * k + 2];
                if (a < 0 || b < 0 || a >= g->n_domains || b >= g->n_domains || f < 0 || f > 3 || a == b)
                    throw Error(FP_ERR_INVALID, "invalid connection in problem " + std::to_string(p));
                P.conns.push_back({a, f, b});
                P.doms[a].bc[f]     = 3;  // Adjacented (Variable2D::set_geometry, variable2d.cpp:25-45)
                P.doms[b].bc[f ^ 1] = 3;
            }
        }
        std::unique_ptr<fp_batch> h(new fp_batch());
        h->b = make_batch(probs, (flags & FP_BATCH_F32) ? 1 : 0);
        if (!(flags & FP_BATCH_NO_AUTOTUNE)) h->b->autotune(0);
        FPB_CUDA(cudaDeviceSynchronize());
        *out = h.release();
    });
}

int fp_batch_solve(fp_batch* b, double* const* fields, const double* const* ghosts, int flags, void* stream, int steps)
{
    return guarded([&] {
        if (!b) throw Error(FP_ERR_INVALID, "null batch");
        if (!(flags & FP_DEVICE)) throw Error(FP_ERR_INVALID, "batched solves take device pointers (FP_DEVICE)");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (flags & FP_BATCH_GRAPH) b->b->solve_graph(fields, ghosts, steps, s);
        else b->b->solve(fields, ghosts, steps, s);
        if (flags & FP_SYNC) FPB_CUDA(cudaStreamSynchronize(s));
    });
}

int fp_batch_residuals(fp_batch* b, const double* const* u, const double* const* rhs, const double* const* ghosts,
                       void* stream, double* rel_residuals)
{
    return guarded([&] {
        if (!b || !u || !rhs || !rel_residuals) throw Error(FP_ERR_INVALID, "null argument");
        b->b->residuals(u, rhs, ghosts, static_cast<cudaStream_t>(stream), rel_residuals);
    });
}

int fp_batch_info(const fp_batch* b, int* n_problems, int* n_domains, int* launch_shape, long long* graph_kernels)
{
    return guarded([&] {
        if (!b) throw Error(FP_ERR_INVALID, "null batch");
        if (n_problems) *n_problems = b->b->n_problems();
        if (n_domains) *n_domains = b->b->n_domains();
        if (launch_shape)
        {
            const BatchTiming t = b->b->timing();
            launch_shape[0]     = t.dst_threads;
            launch_shape[1]     = t.dst_blocks_per_sm;
            launch_shape[2]     = t.chase_threads;
        }
        if (graph_kernels) *graph_kernels = b->b->graph_kernels();
    });
}

int fp_batch_destroy(fp_batch* b)
{
    return guarded([&] { delete b; });
}

}  // extern "C"
