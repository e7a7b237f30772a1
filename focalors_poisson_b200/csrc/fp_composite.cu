// Composite-geometry solve: block elimination over the domain tree with a Schur-complement GMRES at
// every internal node, restating ConcatPoissonSolver2D::solve (pe/concat/concat_solver2d.cpp:101-157)
// and GMRESSolver2D (pe/concat/gmres_solver2d.cpp:39-252) on device buffers.
//
// GMRES works either on the node's interface unknowns (default: the Krylov vectors are the values on
// the node's faces shared with its children, y = P x, solving (I - P A^-1 S) y = P A^-1 b and finishing
// with x = A^-1 b + A^-1 S y), or on full fields exactly like the reference. Each operator apply is
// one rectangle solve of the node plus the children's dense Schur matrices. The orthogonalisation is
// the reference's modified Gram-Schmidt, the small Hessenberg least-squares problem (Givens rotations,
// back substitution) runs on the host in FP64.
#include "fp_batch.h"
#include "fp_composite.h"
#include "fp_ops.cuh"
#include "fp_gmres.cuh"

#include <cublas_v2.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <queue>

namespace fpb
{

namespace
{
inline unsigned grid_for(long long n, int block, int cap = 4096)
{
    long long g = (n + block - 1) / block;
    return (unsigned)std::max(1LL, std::min<long long>(g, cap));
}

}  // namespace

Tree build_tree(int nd, const std::vector<std::array<int, 3>>& conns, int root, int faces)
{
    if (faces != 4 && faces != 6) throw Error(1, "a tree is built over 4 (2D) or 6 (3D) faces");
    if (nd <= 0) throw Error(1, "geometry has no domains");
    std::vector<std::array<int, 6>> adj(nd, {-1, -1, -1, -1, -1, -1});
    for (const auto& c : conns)
    {
        const int a = c[0], loc = c[1], b = c[2];
        if (a < 0 || a >= nd || b < 0 || b >= nd || a == b || loc < 0 || loc >= faces)
            throw Error(1, "invalid connection");
        if ((adj[a][loc] != -1 && adj[a][loc] != b) || (adj[b][loc ^ 1] != -1 && adj[b][loc ^ 1] != a))
            throw Error(1, "a face is connected twice");
        adj[a][loc]     = b;
        adj[b][loc ^ 1] = a;
    }
    // connectivity (Geometry2D::is_single_connected, geometry2d.cpp:109-163) and acyclicity
    long long edges = 0;
    for (int d = 0; d < nd; ++d)
        for (int f = 0; f < faces; ++f) edges += adj[d][f] >= 0;
    edges /= 2;
    {
        std::vector<int> seen(nd, 0);
        std::queue<int>  q;
        q.push(0);
        seen[0] = 1;
        while (!q.empty())
        {
            int u = q.front();
            q.pop();
            for (int f = 0; f < faces; ++f)
                if (adj[u][f] >= 0 && !seen[adj[u][f]])
                {
                    seen[adj[u][f]] = 1;
                    q.push(adj[u][f]);
                }
        }
        for (int d = 0; d < nd; ++d)
            if (!seen[d]) throw Error(1, "Geometry is not single connected");
    }
    if (edges != nd - 1)
        throw Error(1, "geometry adjacency has a cycle; the domain decomposition needs a tree of subdomains");
    Tree t;
    if (root < 0)
    {
        if (nd == 1) root = 0;
        else
        {
            std::vector<int> deg(nd, 0), leaves;
            for (int d = 0; d < nd; ++d)
            {
                for (int f = 0; f < faces; ++f) deg[d] += adj[d][f] >= 0;
                if (deg[d] <= 1) leaves.push_back(d);
            }
            int remaining = nd;
            while (remaining > 2 && !leaves.empty())
            {
                remaining -= (int)leaves.size();
                std::vector<int> next;
                for (int lf : leaves)
                    for (int f = 0; f < faces; ++f)
                        if (adj[lf][f] >= 0 && --deg[adj[lf][f]] == 1) next.push_back(adj[lf][f]);
                leaves.swap(next);
            }
            root = leaves.empty() ? 0 : *std::min_element(leaves.begin(), leaves.end());
        }
    }
    if (root >= nd) throw Error(1, "root index out of range");
    t.root = root;
    t.children.assign(nd, {});
    t.parent.assign(nd, {-1, -1});
    std::vector<int> stack = {root}, par(nd, -2);
    par[root]              = -1;
    while (!stack.empty())
    {
        int u = stack.back();
        stack.pop_back();
        for (int f = 0; f < faces; ++f)
        {
            int v = adj[u][f];
            if (v < 0 || v == par[u]) continue;
            par[v] = u;
            t.children[u].push_back({f, v});
            t.parent[v] = {f ^ 1, u};
            stack.push_back(v);
        }
    }
    std::vector<int> frontier = {root};
    while (!frontier.empty())
    {
        t.levels.push_back(frontier);
        std::vector<int> next;
        for (int d : frontier)
            for (auto& c : t.children[d]) next.push_back(c.second);
        frontier.swap(next);
    }
    return t;
}

Composite::Composite(const std::vector<Domain>& doms, const std::vector<std::array<int, 3>>& conns, int root, int m,
                     double tol, int max_iter, int mode, bool interface_inverse,
                     const std::vector<std::array<int, 2>>& ext)
    : dom_(doms), m_(m), max_iter_(max_iter), mode_(mode), want_inverse_(interface_inverse), tol_(tol)
{
    if (m < 1 || m > 200) throw Error(1, "GMRES restart length m must be in [1, 200]");
    if (max_iter < 1) throw Error(1, "maxIter must be positive");
    const int nd = (int)dom_.size();
    tree_        = build_tree(nd, conns, root);
    for (const auto& c : conns)
    {
        Domain &a = dom_[c[0]], &b = dom_[c[2]];
        a.bc[c[1]]     = BC_ADJACENTED;
        b.bc[c[1] ^ 1] = BC_ADJACENTED;
        const bool xdir = c[1] < 2;
        if (xdir ? (a.ny != b.ny) : (a.nx != b.nx))
            throw Error(1, "connected domains must share the interface length");
    }
    temp_.resize(nd);
    for (int d = 0; d < nd; ++d)
        if (d != tree_.root) temp_[d].alloc(dom_[d].cells() * sizeof(double));
    node_.resize(nd);
    for (int d = 0; d < nd; ++d)
    {
        Node& nd_ = node_[d];
        int   off = 0;
        for (auto& c : tree_.children[d])
        {
            Link L;
            L.loc   = c.first;
            L.child = c.second;
            L.cn    = edge_length(L.loc, dom_[d].nx, dom_[d].ny);
            L.off   = off;
            off += L.cn;
            nd_.kids.push_back(std::move(L));
        }
        if (d == tree_.root)
            for (size_t q = 0; q < ext.size(); ++q)  // children in other parts: no local domain, Schur matrix later
            {
                const auto& e = ext[q];
                if (e[0] < 0 || e[0] > 3) throw Error(1, "external child face out of range");
                if (q > 0 && e[0] <= ext[q - 1][0]) throw Error(1, "external children must be given in face order");
                for (const auto& k : nd_.kids)
                    if (k.loc == e[0]) throw Error(1, "external child on a connected face");
                if (e[1] != edge_length(e[0], dom_[d].nx, dom_[d].ny))
                    throw Error(1, "external child interface length differs from the root's face");
                dom_[d].bc[e[0]] = BC_ADJACENTED;
                Link L;
                L.loc   = e[0];
                L.child = -1;
                L.cn    = e[1];
                L.off   = off;
                off += L.cn;
                nd_.kids.push_back(std::move(L));
                ++n_ext_;
            }
        if (nd_.kids.empty()) continue;
        nd_.n_if = off;
        nd_.n    = (mode_ == GMRES_FULLFIELD) ? dom_[d].cells() : (long long)off;
        nd_.R.alloc(dom_[d].cells() * sizeof(double));
    }
    rect_.resize(nd);  // after the external children's faces became Adjacented
    for (int d = 0; d < nd; ++d)
        rect_[d].reset(new DevRect<double>(dom_[d].nx, dom_[d].ny, dom_[d].hx, dom_[d].hy, dom_[d].bc));
    red_.alloc((kRedBlocks + 8) * sizeof(double));
    FPB_CUDA(cudaMemset(red_.get(), 0, red_.bytes()));
    set_parameter(m, tol, max_iter);
}

// Schur matrices and interface inverses: fp_composite_create builds them through prepare() for a geometry
// outside the spectral path, so that no solve pays for them; a solve that still finds them missing (a
// geometry that left the spectral path later) builds them first.
void Composite::ensure_built()
{
    if (built_) return;
    build_schur();
    if (want_inverse_ && mode_ == GMRES_INTERFACE)
        for (int d = 0; d < (int)dom_.size(); ++d)
            if (!node_[d].kids.empty() && node_[d].n_if <= kMaxInverse) build_interface_inverse(d);
    built_ = true;
}

Composite::~Composite()
{
    drop_gmres_graphs();
    if (gm_host_) cudaFreeHost(gm_host_);
}

void Composite::set_parameter(int m, double tol, int max_iter)
{
    if (m < 1 || m > 200) throw Error(1, "GMRES restart length m must be in [1, 200]");
    const bool rebuild = (m != m_ || tol != tol_ || max_iter != max_iter_);
    m_                 = m;
    tol_               = tol;
    max_iter_          = max_iter;
    gm_graph_.resize(node_.size(), nullptr);
    drop_gmres_graphs();  // they hold the buffers below and the parameters
    for (auto& nd : node_)
    {
        if (nd.kids.empty()) continue;
        nd.V.alloc((size_t)(m_ + 1) * nd.n * sizeof(double));
        nd.w.alloc(nd.n * sizeof(double));
        nd.r.alloc(nd.n * sizeof(double));
        nd.x.alloc(nd.n * sizeof(double));
        nd.b.alloc(nd.n * sizeof(double));
        nd.hcol.alloc((m_ + 2) * sizeof(double));
        nd.tmp.alloc(64 * sizeof(double) + (size_t)(m_ + 1) * sizeof(double));
    }
    // Nested GMRES tolerances enter the Schur matrices of internal children, so the reference rebuilds
    // its solver map when parameters change (concat_solver2d.cpp:7-17); do the same.
    if (rebuild)
    {
        bool nested = false;
        for (int d = 0; d < (int)node_.size(); ++d)
            if (d != tree_.root && !node_[d].kids.empty()) nested = true;
        bool built = false;
        for (auto& nd : node_)
            for (auto& L : nd.kids) built |= L.S.get() != nullptr;
        if (nested && built) build_schur();
    }
}

double Composite::dot(const double* a, const double* b, long long n, bool sqrt_, cudaStream_t s, double* dev_out)
{
    double*   partials = red_.as<double>();
    unsigned* ticket   = reinterpret_cast<unsigned*>(partials + kRedBlocks);
    k_dot<<<grid_for(n, kRedThreads, kRedBlocks), kRedThreads, 0, s>>>(a, b, n, partials, ticket, dev_out,
                                                                      sqrt_ ? 1 : 0);
    FPB_CHECK_LAUNCH();
    return 0.0;
}

void Composite::schur_apply_into(int d, const double* vec, bool vec_is_field, double* R, cudaStream_t s)
{
    const Domain& D = dom_[d];
    for (const Link& L : node_[d].kids)
    {
        const double* v      = vec_is_field ? vec + edge_index(L.loc, D.nx, D.ny, 0) : vec + L.off;
        long long     stride = 1;
        if (vec_is_field && L.loc >= 2) stride = D.ny;
        const int warps = 8;
        k_schur_matvec<double><<<(L.cn + warps - 1) / warps, warps * 32, 0, s>>>(L.S.as<double>(), L.cn, v, stride, R,
                                                                                D.nx, D.ny, L.loc);
        FPB_CHECK_LAUNCH();
    }
}

void Composite::rect_solve(int d, double* f, long long batch, cudaStream_t s) const
{
    if (mixed_) rect_[d]->solve_mixed(f, batch, s);
    else rect_[d]->solve(f, batch, s);
}

void Composite::afun(int d, const double* v, double* out, cudaStream_t s)
{
    Node&         N = node_[d];
    const Domain& D = dom_[d];
    double*       R = N.R.as<double>();
    FPB_CUDA(cudaMemsetAsync(R, 0, D.cells() * sizeof(double), s));
    schur_apply_into(d, v, mode_ == GMRES_FULLFIELD, R, s);
    rect_[d]->solve(R, 1, s);
    if (mode_ == GMRES_FULLFIELD)
    {
        k_sub<<<grid_for(N.n, 256), 256, 0, s>>>(out, v, R, N.n);
        FPB_CHECK_LAUNCH();
        return;
    }
    for (const Link& L : N.kids)
    {
        k_edge_sub<double><<<grid_for(L.cn, 128), 128, 0, s>>>(out + L.off, v + L.off, R, D.nx, D.ny, L.loc);
        FPB_CHECK_LAUNCH();
    }
}

void Composite::node_solve(int d, double* f, cudaStream_t s, GmresInfo* info)
{
    Node& N = node_[d];
    if (N.kids.empty())
    {
        rect_solve(d, f, 1, s);
        return;
    }
    if (mixed_ && N.has_inv)
    {
        // inner solve of iterative refinement: y = X g, f = A^-1 b + A^-1 S y, no residual test
        const Domain& D = dom_[d];
        double *g = N.b.as<double>(), *y = N.x.as<double>(), *Z = N.Z.as<double>();
        rect_solve(d, f, 1, s);
        for (const Link& L : N.kids)
        {
            k_edge_gather<double><<<grid_for(L.cn, 128), 128, 0, s>>>(g + L.off, f, D.nx, D.ny, L.loc);
            FPB_CHECK_LAUNCH();
        }
        const int warps = 8;
        k_dense_matvec<<<(N.n_if + warps - 1) / warps, warps * 32, 0, s>>>(N.X.as<double>(), N.n_if, g, y, 0);
        FPB_CHECK_LAUNCH();
        FPB_CUDA(cudaMemsetAsync(Z, 0, D.cells() * sizeof(double), s));
        schur_apply_into(d, y, false, Z, s);
        rect_solve(d, Z, 1, s);
        k_add<double><<<grid_for(D.cells(), 256), 256, 0, s>>>(f, Z, D.cells());
        FPB_CHECK_LAUNCH();
        if (info) info->iterations += 1;
        return;
    }
    const Domain& D = dom_[d];
    const long long n = N.n;
    double *        x = N.x.as<double>(), *b = N.b.as<double>();

    rect_[d]->solve(f, 1, s);  // b <- A^-1 b (gmres_solver2d.cpp:130)
    if (mode_ == GMRES_FULLFIELD)
        FPB_CUDA(cudaMemcpyAsync(b, f, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else
        for (const Link& L : N.kids)
        {
            k_edge_gather<double><<<grid_for(L.cn, 128), 128, 0, s>>>(b + L.off, f, D.nx, D.ny, L.loc);
            FPB_CHECK_LAUNCH();
        }
    FPB_CUDA(cudaMemcpyAsync(x, b, n * sizeof(double), cudaMemcpyDeviceToDevice, s));

    if (N.has_inv && refine_with_inverse(d, f, s, info)) return;

    // the restart loop (gmres_solver2d.cpp:139-249) as one CUDA graph over the node's buffers (fp_gmres.cuh)
    if (!gm_graph_[d]) build_gmres_graph(d, s);
    FPB_CUDA(cudaGraphLaunch(gm_graph_[d], s));
    FPB_CUDA(cudaMemcpyAsync(gm_host_, N.st.get(), sizeof(GmState), cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
    const GmState gs = *gm_host_;
    if (gs.err) throw Error(5, "non-finite GMRES value");
    const bool   converged = gs.converged != 0;
    const double last_res  = gs.beta;
    const int    iters = gs.iters, restarts = gs.restarts;
    if (mode_ == GMRES_FULLFIELD)
    {
        FPB_CUDA(cudaMemcpyAsync(f, x, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    else
    {
        double* R = N.R.as<double>();
        FPB_CUDA(cudaMemsetAsync(R, 0, D.cells() * sizeof(double), s));
        schur_apply_into(d, x, false, R, s);
        rect_[d]->solve(R, 1, s);
        k_add<double><<<grid_for(D.cells(), 256), 256, 0, s>>>(f, R, D.cells());
        FPB_CHECK_LAUNCH();
    }
    if (info)
    {
        info->iterations += iters;
        info->restarts += restarts;
        info->residual  = last_res;
        info->converged = info->converged && converged;
    }
}

void Composite::build_gmres_graph(int d, cudaStream_t s)
{
    Node&           N = node_[d];
    const Domain&   D = dom_[d];
    const long long n = N.n;
    const int       m = m_;
    N.vin.alloc(n * sizeof(double));
    N.arr.alloc((size_t)((m + 1) * m + 3 * m + 1) * sizeof(double));
    N.st.alloc(sizeof(GmState));
    GmBuffers B;
    B.V        = N.V.as<double>();
    B.w        = N.w.as<double>();
    B.r        = N.r.as<double>();
    B.x        = N.x.as<double>();
    B.b        = N.b.as<double>();
    B.vin      = N.vin.as<double>();
    B.st       = N.st.as<GmState>();
    B.a.H      = N.arr.as<double>();
    B.a.cs     = B.a.H + (size_t)(m + 1) * m;
    B.a.sn     = B.a.cs + m;
    B.a.g      = B.a.sn + m;
    B.a.y      = B.a.g + (m + 1);
    B.a.hcol   = N.hcol.as<double>();
    B.partials = red_.as<double>();
    B.ticket   = reinterpret_cast<unsigned*>(B.partials + kRedBlocks);
    if (!gm_host_) FPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&gm_host_), sizeof(GmState)));
    // warm-up outside the capture: the rectangle solves' work buffers are allocated on first use
    afun(d, B.x, B.w, s);
    rect_[d]->solve(N.R.as<double>(), 1, s);
    FPB_CUDA(cudaStreamSynchronize(s));
    const bool iface = mode_ == GMRES_INTERFACE;
    gm_graph_[d] = capture_gmres(
        n, m, tol_, max_iter_, iface, B, [&](const double* in, double* out, cudaStream_t q) { afun(d, in, out, q); },
        [&](cudaStream_t q) {
            if (!iface) return;
            // the reference's test is on the full-field residual A^-1 S rho(y) of the iterate (gmres_solver2d.cpp:149-160)
            double* R = N.R.as<double>();
            FPB_CUDA(cudaMemsetAsync(R, 0, D.cells() * sizeof(double), q));
            schur_apply_into(d, B.r, false, R, q);
            rect_[d]->solve(R, 1, q);
            dot(R, R, D.cells(), true, q, B.a.hcol + m);
        },
        [&](const double* a, const double* b, long long len, bool sq, double* out, cudaStream_t q) {
            dot(a, b, len, sq, q, out);
        });
}

void Composite::drop_gmres_graphs()
{
    for (auto& g : gm_graph_)
        if (g)
        {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

namespace
{
struct Cublas
{
    cublasHandle_t h = nullptr;
    Cublas()
    {
        if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) throw Error(2, "cublasCreate failed");
    }
    ~Cublas()
    {
        if (h) cublasDestroy(h);
    }
    // C = A B for row-major n x n matrices (column-major view: C^T = B^T A^T)
    void gemm(const double* A, const double* B, double* C, int n)
    {
        const double one = 1.0, zero = 0.0;
        if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, B, n, A, n, &zero, C, n) != CUBLAS_STATUS_SUCCESS)
            throw Error(2, "cublasDgemm failed");
    }
};
}  // namespace

// Dense interface operator M = I - P A^-1 E S of node d (column c = response on all of d's interface
// cells to the c-th Schur column placed on its edge, one batched rectangle solve per block of columns)
// and its inverse by the Newton-Schulz iteration X <- X (2I - M X), X_0 = M^T / (|M|_1 |M|_inf), which
// converges for any nonsingular M. Only GEMMs (cuBLAS) and small kernels.
void Composite::build_interface_inverse(int d)
{
    Node&           N     = node_[d];
    const Domain&   D     = dom_[d];
    const int       n     = N.n_if;
    const long long cells = D.cells();
    cudaStream_t    s     = 0;
    DevBuf          M((size_t)n * n * sizeof(double)), X((size_t)n * n * sizeof(double)), P((size_t)n * n * sizeof(double));
    const long long nb    = std::max(1LL, std::min<long long>(n, (512LL << 20) / (cells * 8)));
    DevBuf          work((size_t)nb * cells * sizeof(double));
    for (const Link& L : N.kids)
        for (int c0 = 0; c0 < L.cn; c0 += (int)nb)
        {
            const int cnt = (int)std::min<long long>(nb, L.cn - c0);
            FPB_CUDA(cudaMemsetAsync(work.get(), 0, (size_t)cnt * cells * sizeof(double), s));
            k_edge_scatter_col<<<grid_for((long long)cnt * L.cn, 256), 256, 0, s>>>(
                work.as<double>(), cells, D.nx, D.ny, L.loc, L.S.as<double>(), L.cn, c0, cnt);
            FPB_CHECK_LAUNCH();
            rect_[d]->solve(work.as<double>(), cnt, s);
            for (const Link& Lo : N.kids)
            {
                k_edge_gather_col<<<grid_for((long long)cnt * Lo.cn, 256), 256, 0, s>>>(
                    M.as<double>(), n, Lo.off, work.as<double>(), cells, D.nx, D.ny, Lo.loc, Lo.cn, L.off + c0, cnt);
                FPB_CHECK_LAUNCH();
            }
        }
    const long long nn = (long long)n * n;
    k_identity_minus<<<grid_for(nn, 256, 1 << 30), 256, 0, s>>>(M.as<double>(), n);
    FPB_CHECK_LAUNCH();
    DevBuf sums(2 * (size_t)n * sizeof(double));
    k_abs_sums<<<grid_for(n, 128), 128, 0, s>>>(M.as<double>(), n, sums.as<double>(), sums.as<double>() + n);
    FPB_CHECK_LAUNCH();
    std::vector<double> hs(2 * (size_t)n);
    FPB_CUDA(cudaMemcpy(hs.data(), sums.get(), hs.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const double ninf = *std::max_element(hs.begin(), hs.begin() + n);
    const double n1   = *std::max_element(hs.begin() + n, hs.end());
    if (!(ninf > 0) || !std::isfinite(ninf * n1)) throw Error(5, "interface operator is zero or not finite");
    k_scaled_transpose<<<grid_for(nn, 256, 1 << 30), 256, 0, s>>>(X.as<double>(), M.as<double>(), n, 1.0 / (ninf * n1));
    FPB_CHECK_LAUNCH();
    Cublas    cb;
    double*   partials = red_.as<double>();
    unsigned* ticket   = reinterpret_cast<unsigned*>(partials + kRedBlocks);
    double*   out      = partials + kRedBlocks + 2;
    double    prev     = 1e300;
    bool      ok       = false;
    work.release();
    DevBuf Xn((size_t)n * n * sizeof(double));
    for (int it = 0; it < 200; ++it)
    {
        cb.gemm(M.as<double>(), X.as<double>(), P.as<double>(), n);  // P = M X
        k_identity_residual<<<kRedBlocks, kRedThreads, 0, s>>>(P.as<double>(), n, partials, ticket, out);
        FPB_CHECK_LAUNCH();
        double err2 = 0;
        FPB_CUDA(cudaMemcpy(&err2, out, sizeof(double), cudaMemcpyDeviceToHost));
        const double err = std::sqrt(err2);  // ||I - M X||_F
        if (!std::isfinite(err)) break;
        if (err < 1e-13 * std::sqrt((double)n) || (err < 1e-6 && err > 0.5 * prev))
        {
            ok = err < 1e-6;  // converged, or stalled at round-off
            break;
        }
        prev = err;
        k_two_identity_minus<<<grid_for(nn, 256, 1 << 30), 256, 0, s>>>(P.as<double>(), n);  // P = 2I - M X
        FPB_CHECK_LAUNCH();
        cb.gemm(X.as<double>(), P.as<double>(), Xn.as<double>(), n);  // X <- X (2I - M X)
        std::swap(X, Xn);
    }
    FPB_CUDA(cudaDeviceSynchronize());
    if (ok)
    {
        N.X       = std::move(X);
        N.Z.alloc(cells * sizeof(double));
        N.has_inv = true;
    }
}

// Interface solve with the precomputed inverse X of M = I - P A^-1 S, accepted by the reference's test:
// y = X g; Z = A^-1 S y; interface residual rho = g - M y = g - y + P Z; accept when the full-field
// residual |A^-1 S rho| < tol, otherwise y += X rho and repeat (at most 4 times). On success
// f = A^-1 b + Z. Returns false (f untouched beyond b = A^-1 b) if it did not converge; the caller then
// runs GMRES from scratch.
bool Composite::refine_with_inverse(int d, double* f, cudaStream_t s, GmresInfo* info)
{
    Node&         N = node_[d];
    const Domain& D = dom_[d];
    const int     n = N.n_if;
    double *g = N.b.as<double>(), *y = N.x.as<double>(), *rho = N.r.as<double>(), *Z = N.Z.as<double>(),
           *R = N.R.as<double>(), *hcol = N.hcol.as<double>();
    const int warps = 8;
    k_dense_matvec<<<(n + warps - 1) / warps, warps * 32, 0, s>>>(N.X.as<double>(), n, g, y, 0);
    FPB_CHECK_LAUNCH();
    double beta = 0, prev = 1e300;
    for (int it = 0; it < 6; ++it)
    {
        FPB_CUDA(cudaMemsetAsync(Z, 0, D.cells() * sizeof(double), s));
        schur_apply_into(d, y, false, Z, s);
        rect_[d]->solve(Z, 1, s);
        for (const Link& L : N.kids)
        {
            k_interface_residual<<<grid_for(L.cn, 128), 128, 0, s>>>(rho + L.off, g + L.off, y + L.off, Z, D.nx, D.ny,
                                                                   L.loc, L.cn);
            FPB_CHECK_LAUNCH();
        }
        FPB_CUDA(cudaMemsetAsync(R, 0, D.cells() * sizeof(double), s));
        schur_apply_into(d, rho, false, R, s);
        rect_[d]->solve(R, 1, s);
        dot(R, R, D.cells(), true, s, hcol);
        FPB_CUDA(cudaMemcpyAsync(&beta, hcol, sizeof(double), cudaMemcpyDeviceToHost, s));
        FPB_CUDA(cudaStreamSynchronize(s));
        if (!std::isfinite(beta)) break;
        if (info) info->iterations += 1;
        // accept below tol; also accept (reported as not converged) once refinement stops gaining, which
        // happens only when tol is below the round-off floor of the problem
        const bool stalled = it > 0 && beta > 0.5 * prev;
        if (beta < tol_ || stalled)
        {
            k_add<double><<<grid_for(D.cells(), 256), 256, 0, s>>>(f, Z, D.cells());
            FPB_CHECK_LAUNCH();
            if (info)
            {
                info->residual  = beta;
                info->converged = info->converged && beta < tol_;
            }
            return true;
        }
        prev = beta;
        k_dense_matvec<<<(n + warps - 1) / warps, warps * 32, 0, s>>>(N.X.as<double>(), n, rho, y, 1);
        FPB_CHECK_LAUNCH();
    }
    // not converged: restart plain GMRES from the gathered right-hand side
    FPB_CUDA(cudaMemcpyAsync(y, g, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return false;
}

// Schur matrix of an internal child c whose own children are all leaves: the subtree (c and its leaves,
// c's face toward d Adjacented) is a depth-1 tree, which the spectral batched solver covers when its
// boundary types allow. K copies of the subtree are solved at once, copy q carrying the unit impulse at
// interface cell i0 + q; the responses on c's interface row are the matrix's columns. Returns false (and
// builds nothing) when the subtree is outside the spectral solver's scope.
bool Composite::schur_by_spectral(Link& L, cudaStream_t s)
{
    const int c = L.child;
    std::vector<int> map = {c};
    for (auto& k : tree_.children[c])
    {
        if (!node_[k.second].kids.empty()) return false;
        map.push_back(k.second);
    }
    BatchProblemDesc desc;
    for (int g : map) desc.doms.push_back(dom_[g]);  // Adjacented faces already marked, c's parent face included
    for (size_t q = 1; q < map.size(); ++q) desc.conns.push_back({0, tree_.children[c][q - 1].first, (int)q});
    long long sub_cells = 0;
    for (int g : map) sub_cells += dom_[g].cells();
    const long long K = std::max(1LL, std::min<long long>(L.cn, (4LL << 30) / (sub_cells * 8 * 4)));
    std::unique_ptr<BatchBase> b;
    try
    {
        b = make_batch(std::vector<BatchProblemDesc>((size_t)K, desc), 0);
    }
    catch (const Error& e)
    {
        if (e.code != 3) throw;
        return false;
    }
    b->autotune(s);
    const Domain& C    = dom_[c];
    const int     face = L.loc ^ 1;  // c's face toward its parent
    std::vector<DevBuf> bufs(map.size());
    for (size_t q = 0; q < map.size(); ++q) bufs[q].alloc((size_t)K * dom_[map[q]].cells() * sizeof(double));
    std::vector<double*> ptrs;
    for (long long k = 0; k < K; ++k)
        for (size_t q = 0; q < map.size(); ++q) ptrs.push_back(bufs[q].as<double>() + k * dom_[map[q]].cells());
    for (int i0 = 0; i0 < L.cn; i0 += (int)K)
    {
        const int cnt = (int)std::min<long long>(K, L.cn - i0);
        for (size_t q = 0; q < map.size(); ++q)
            FPB_CUDA(cudaMemsetAsync(bufs[q].get(), 0, bufs[q].bytes(), s));
        k_impulses<double><<<grid_for(cnt, 128), 128, 0, s>>>(bufs[0].as<double>(), C.nx, C.ny, face, i0, cnt);
        FPB_CHECK_LAUNCH();
        b->solve(ptrs.data(), nullptr, 0, s);
        k_impulse_extract<double><<<grid_for((long long)cnt * L.cn, 256), 256, 0, s>>>(
            bufs[0].as<double>(), C.nx, C.ny, face, L.S.as<double>(), L.cn, i0, cnt);
        FPB_CHECK_LAUNCH();
    }
    // the batched solve scales its right-hand side by hx^2 (the reference's assembly); the Schur matrix is
    // the response to the unscaled impulse
    k_scale<<<grid_for((long long)L.cn * L.cn, 256), 256, 0, s>>>(L.S.as<double>(), 1.0 / (C.hx * C.hx),
                                                                   (long long)L.cn * L.cn);
    FPB_CHECK_LAUNCH();
    FPB_CUDA(cudaStreamSynchronize(s));
    return true;
}

// One Schur matrix (SchurMat2D_*::construct, schur_mat2d.cpp:5-106): column i = the child's response along its
// face toward the parent to a unit impulse at cell i of that face; by batched rectangle solves for a leaf, by
// the spectral closed form where it applies, else by one subtree solve per impulse.
void Composite::link_schur(Link& L, cudaStream_t s)
{
    const int       c     = L.child;
    const Domain&   C     = dom_[c];
    const int       face  = L.loc ^ 1;  // child's face toward its parent
    const long long cells = C.cells();
    L.S.alloc((size_t)L.cn * L.cn * sizeof(double));
    const bool leaf = node_[c].kids.empty();
    if (!leaf && mode_ != GMRES_FULLFIELD && schur_by_spectral(L, s)) return;
    long long nb = leaf ? std::max(1LL, std::min<long long>(L.cn, (512LL << 20) / (cells * 8))) : 1;
    DevBuf    work((size_t)nb * cells * sizeof(double));
    for (int i0 = 0; i0 < L.cn; i0 += (int)nb)
    {
        const int cnt = (int)std::min<long long>(nb, L.cn - i0);
        FPB_CUDA(cudaMemsetAsync(work.get(), 0, (size_t)cnt * cells * sizeof(double), s));
        k_impulses<double><<<grid_for(cnt, 128), 128, 0, s>>>(work.as<double>(), C.nx, C.ny, face, i0, cnt);
        FPB_CHECK_LAUNCH();
        if (leaf) rect_[c]->solve(work.as<double>(), cnt, s);
        else
            for (int b = 0; b < cnt; ++b) node_solve(c, work.as<double>() + (size_t)b * cells, s, nullptr);
        k_impulse_extract<double><<<grid_for((long long)cnt * L.cn, 256), 256, 0, s>>>(
            work.as<double>(), C.nx, C.ny, face, L.S.as<double>(), L.cn, i0, cnt);
        FPB_CHECK_LAUNCH();
    }
    FPB_CUDA(cudaStreamSynchronize(s));
}

void Composite::build_schur()
{
    cudaStream_t s = 0;
    for (auto lv = tree_.levels.rbegin(); lv != tree_.levels.rend(); ++lv)
        for (int d : *lv)
            for (Link& L : node_[d].kids)
            {
                if (L.child >= 0) link_schur(L, s);
                else if (!L.S.get()) throw Error(1, "external child's Schur matrix not set");
            }
}

void Composite::solve(double* const* fields, const double* const* ghosts, cudaStream_t s, GmresInfo* info)
{
    mixed_ = false;
    assemble(fields, ghosts, s);
    eliminate(fields, s, info);
}

void Composite::assemble(double* const* fields, const double* const* ghosts, cudaStream_t s)
{
    const int nd = (int)dom_.size();
    for (int d = 0; d < nd; ++d)
    {
        const Domain& D = dom_[d];
        AssembleArgs  a;
        a.nx = D.nx;
        a.ny = D.ny;
        a.hx = D.hx;
        a.hy = D.hy;
        for (int f = 0; f < 4; ++f)
        {
            a.bc[f]    = D.bc[f];
            a.ghost[f] = ghosts ? ghosts[4 * d + f] : nullptr;
        }
        k_assemble_scale<double><<<grid_for(D.cells(), 256, 1 << 30), 256, 0, s>>>(fields[d], a);
        FPB_CHECK_LAUNCH();
    }
}

void Composite::eliminate(double* const* fields, cudaStream_t s, GmresInfo* info, const double* const* child_edges,
                          double* const* edges_out)
{
    ensure_built();
    auto bond = [&](double* dst, int dd, int loc, const double* src, int sd) {
        const Domain &A = dom_[dd], &B = dom_[sd];
        k_bond_add<double><<<grid_for(edge_length(loc, A.nx, A.ny), 128), 128, 0, s>>>(dst, A.nx, A.ny, loc, -1.0, src,
                                                                                     B.nx, B.ny);
        FPB_CHECK_LAUNCH();
    };
    const auto& T = tree_;
    for (int l = (int)T.levels.size() - 1; l >= 1; --l)
    {
        for (int d : T.levels[l])
        {
            double* td = temp_[d].as<double>();
            FPB_CUDA(cudaMemcpyAsync(td, fields[d], dom_[d].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
            for (auto& c : T.children[d])
            {
                bond(td, d, c.first, temp_[c.second].as<double>(), c.second);
                bond(fields[d], d, c.first, temp_[c.second].as<double>(), c.second);
            }
        }
        for (int d : T.levels[l]) node_solve(d, temp_[d].as<double>(), s, nullptr);
    }
    for (auto& c : T.children[T.root]) bond(fields[T.root], T.root, c.first, temp_[c.second].as<double>(), c.second);
    if (n_ext_ > 0 && !child_edges) throw Error(1, "a root part needs its external children's interface values");
    int e = 0;
    for (const Link& L : node_[T.root].kids)  // children in other parts: their solved copies' edges
        if (L.child < 0) edge_axpy(fields[T.root], T.root, L.loc, -1.0, child_edges[e++], s);
    node_solve(T.root, fields[T.root], s, info);
    e = 0;
    for (const Link& L : node_[T.root].kids)
        if (L.child < 0 && edges_out)
        {
            const Domain& R = dom_[T.root];
            k_edge_gather<double><<<grid_for(L.cn, 128), 128, 0, s>>>(edges_out[e++], fields[T.root], R.nx, R.ny, L.loc);
            FPB_CHECK_LAUNCH();
        }
    for (size_t l = 1; l < T.levels.size(); ++l)
    {
        for (int d : T.levels[l]) bond(fields[d], d, T.parent[d].first, fields[T.parent[d].second], T.parent[d].second);
        for (int d : T.levels[l]) node_solve(d, fields[d], s, nullptr);
    }
}

int Composite::solve_ir(double* const* fields, const double* const* ghosts, cudaStream_t s, double rel_tol,
                        int max_refine, double* rel_change, GmresInfo* info, bool inner_fp32)
{
    ensure_ir_workspace();
    mixed_ = false;
    assemble(fields, ghosts, s);
    return refine(fields, s, rel_tol, max_refine, rel_change, info, inner_fp32);
}

int Composite::refine(double* const* fields, cudaStream_t s, double rel_tol, int max_refine, double* rel_change,
                      GmresInfo* info, bool inner_fp32)
{
    const int nd = (int)dom_.size();
    for (int d = 0; d < nd; ++d)
    {
        FPB_CUDA(cudaMemcpyAsync(fs_[d].get(), fields[d], dom_[d].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
        FPB_CUDA(cudaMemsetAsync(u_[d].get(), 0, dom_[d].cells() * sizeof(double), s));
    }
    std::vector<double> hs(2 * (size_t)nd);
    double              change = 1.0;
    int                 steps  = 0;
    for (; steps < max_refine;)
    {
        mixed_ = inner_fp32;
        eliminate(fields, s, info);  // fields: residual in, correction out
        mixed_ = false;
        ++steps;
        for (int d = 0; d < nd; ++d)
        {
            k_add<double><<<grid_for(dom_[d].cells(), 256), 256, 0, s>>>(u_[d].as<double>(), fields[d], dom_[d].cells());
            FPB_CHECK_LAUNCH();
            dot(fields[d], fields[d], dom_[d].cells(), false, s, sums_.as<double>() + 2 * d);
            dot(u_[d].as<double>(), u_[d].as<double>(), dom_[d].cells(), false, s, sums_.as<double>() + 2 * d + 1);
        }
        FPB_CUDA(cudaMemcpyAsync(hs.data(), sums_.get(), hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        FPB_CUDA(cudaStreamSynchronize(s));
        double en = 0, un = 0;
        for (int d = 0; d < nd; ++d)
        {
            en += hs[2 * d];
            un += hs[2 * d + 1];
        }
        if (!std::isfinite(en) || !std::isfinite(un)) throw Error(5, "non-finite value in iterative refinement");
        const double last = change;
        change            = un > 0 ? std::sqrt(en / un) : 0.0;
        // stop when this correction is below tol, or when the observed contraction rate says the error left
        // after applying it (about change * change / last) is
        if (change <= rel_tol || (steps >= 2 && last > 0 && change * (change / last) <= rel_tol)) break;
        std::vector<double*>       r(nd);
        std::vector<const double*> fsp(nd), up(nd);
        for (int d = 0; d < nd; ++d)
        {
            r[d]   = fields[d];
            fsp[d] = fs_[d].as<double>();
            up[d]  = u_[d].as<double>();
        }
        residual_into(r.data(), fsp.data(), up.data(), s);  // fields <- fs - A u
    }
    for (int d = 0; d < nd; ++d)
        FPB_CUDA(cudaMemcpyAsync(fields[d], u_[d].get(), dom_[d].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (rel_change) *rel_change = change;
    return steps;
}

// The operator ConcatPoissonSolver2D::solve inverts is A u = H (f + b(ghosts)), H = diag(hx_d^2) per domain,
// A the composite 5-point operator of k_composite_residual. A is symmetric: inside a domain the x and y
// stencils are symmetric for every boundary type (Dirichlet ghosts move to the right-hand side, Neumann
// mirrors, periodic wraps), and every interface couples the two adjacent cells with coefficient 1 in both
// equations (bond_add with coefficient -1 on both sides, pe/concat/concat_solver2d.cpp:101-157). The map
// f -> u is therefore A^-1 H, and its transpose is H A^-1: the same elimination applied to the unscaled,
// unassembled vector, then scaled by hx_d^2. Without any Dirichlet face A is singular and the forward solve
// picks one particular solution, which has no such transpose: refused.
void Composite::require_nonsingular() const
{
    for (const Domain& D : dom_)
        for (int f = 0; f < 4; ++f)
            if (D.bc[f] == 0) return;
    throw Error(3, "adjoint solve needs a Dirichlet face: the composite operator is singular");
}

void Composite::scale_by_h2(double* const* fields, cudaStream_t s)
{
    for (size_t d = 0; d < dom_.size(); ++d)
    {
        k_scale<<<grid_for(dom_[d].cells(), 256), 256, 0, s>>>(fields[d], dom_[d].hx * dom_[d].hx, dom_[d].cells());
        FPB_CHECK_LAUNCH();
    }
}

// The elimination's GMRES tolerance is absolute and sized for the hx^2-scaled right-hand sides of a forward
// solve, so the unscaled input is brought to that scale first (c = hx^2 of the root) and the result back.
void Composite::solve_adjoint(double* const* fields, cudaStream_t s, GmresInfo* info)
{
    require_nonsingular();
    mixed_         = false;
    const double c = dom_[tree_.root].hx * dom_[tree_.root].hx;
    for (size_t d = 0; d < dom_.size(); ++d)
    {
        k_scale<<<grid_for(dom_[d].cells(), 256), 256, 0, s>>>(fields[d], c, dom_[d].cells());
        FPB_CHECK_LAUNCH();
    }
    eliminate(fields, s, info);
    for (size_t d = 0; d < dom_.size(); ++d)
    {
        k_scale<<<grid_for(dom_[d].cells(), 256), 256, 0, s>>>(fields[d], dom_[d].hx * dom_[d].hx / c, dom_[d].cells());
        FPB_CHECK_LAUNCH();
    }
}

void Composite::scale_fields(double* const* fields, bool by_h2, cudaStream_t s)
{
    for (size_t d = 0; d < dom_.size(); ++d)
    {
        const double h2 = dom_[d].hx * dom_[d].hx;
        k_scale<<<grid_for(dom_[d].cells(), 256), 256, 0, s>>>(fields[d], by_h2 ? h2 : 1.0 / h2, dom_[d].cells());
        FPB_CHECK_LAUNCH();
    }
}

int Composite::solve_adjoint_ir(double* const* fields, cudaStream_t s, double rel_tol, int max_refine,
                                double* rel_change, GmresInfo* info, bool inner_fp32)
{
    require_nonsingular();
    ensure_ir_workspace();
    mixed_    = false;
    const int steps = refine(fields, s, rel_tol, max_refine, rel_change, info, inner_fp32);
    scale_by_h2(fields, s);
    return steps;
}

void Composite::ensure_ir_workspace()
{
    const int nd = (int)dom_.size();
    if ((int)fs_.size() == nd) return;
    fs_.resize(nd);
    u_.resize(nd);
    for (int d = 0; d < nd; ++d)
    {
        fs_[d].alloc(dom_[d].cells() * sizeof(double));
        u_[d].alloc(dom_[d].cells() * sizeof(double));
    }
    sums_.alloc(2 * (size_t)nd * sizeof(double));
}

void Composite::residual_into(double* const* r, const double* const* fs, const double* const* u, cudaStream_t s)
{
    const int nd = (int)dom_.size();
    for (int d = 0; d < nd; ++d)
    {
        const Domain& D = dom_[d];
        ResidualArgs  a{};
        a.nx = D.nx;
        a.ny = D.ny;
        a.r2 = D.hx * D.hx / D.hy / D.hy;
        for (int f = 0; f < 4; ++f)
        {
            a.bc[f] = D.bc[f];
            a.nb[f] = nullptr;
        }
        for (auto& c : tree_.children[d])
        {
            a.nb[c.first]   = u[c.second];
            a.nbnx[c.first] = dom_[c.second].nx;
            a.nbny[c.first] = dom_[c.second].ny;
        }
        if (tree_.parent[d].second >= 0)
        {
            const int f = tree_.parent[d].first, p = tree_.parent[d].second;
            a.nb[f]     = u[p];
            a.nbnx[f]   = dom_[p].nx;
            a.nbny[f]   = dom_[p].ny;
        }
        k_composite_residual<<<grid_for(D.cells(), 256, 1 << 30), 256, 0, s>>>(r[d], fs[d], u[d], a);
        FPB_CHECK_LAUNCH();
    }
}

double Composite::residual_norm(const double* const* u, const double* const* rhs, const double* const* ghosts,
                                cudaStream_t s)
{
    const int nd = (int)dom_.size();
    ensure_ir_workspace();
    std::vector<double*>       fsp(nd), rp(nd);
    std::vector<const double*> fsc(nd);
    for (int d = 0; d < nd; ++d)
    {
        fsp[d] = fs_[d].as<double>();
        fsc[d] = fsp[d];
        rp[d]  = u_[d].as<double>();  // residual scratch
        FPB_CUDA(cudaMemcpyAsync(fsp[d], rhs[d], dom_[d].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    assemble(fsp.data(), ghosts, s);
    residual_into(rp.data(), fsc.data(), u, s);
    for (int d = 0; d < nd; ++d)
    {
        dot(rp[d], rp[d], dom_[d].cells(), false, s, sums_.as<double>() + 2 * d);
        dot(fsp[d], fsp[d], dom_[d].cells(), false, s, sums_.as<double>() + 2 * d + 1);
    }
    std::vector<double> hs(2 * (size_t)nd);
    FPB_CUDA(cudaMemcpyAsync(hs.data(), sums_.get(), hs.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    FPB_CUDA(cudaStreamSynchronize(s));
    double rn = 0, fn = 0;
    for (int d = 0; d < nd; ++d)
    {
        rn += hs[2 * d];
        fn += hs[2 * d + 1];
    }
    return fn > 0 ? std::sqrt(rn / fn) : std::sqrt(rn);
}

namespace
{
// field.edge(loc)[k] += a * v[k]  (field2::bond_add with a neighbour's edge given as a vector)
__global__ void k_edge_axpy(double* __restrict__ field, int nx, int ny, int loc, double a, const double* __restrict__ v)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= edge_length(loc, nx, ny)) return;
    field[edge_index(loc, nx, ny, k)] += a * v[k];
}
}  // namespace

void Composite::edge_axpy(double* field, int d, int loc, double a, const double* v, cudaStream_t s)
{
    const Domain& D = dom_[d];
    k_edge_axpy<<<grid_for(edge_length(loc, D.nx, D.ny), 128), 128, 0, s>>>(field, D.nx, D.ny, loc, a, v);
    FPB_CHECK_LAUNCH();
}

void Composite::set_external_schur(int k, const double* S_dev)
{
    int e = 0;
    for (Link& L : node_[tree_.root].kids)
        if (L.child < 0 && e++ == k)
        {
            L.S.alloc((size_t)L.cn * L.cn * sizeof(double));
            FPB_CUDA(cudaMemcpy(L.S.get(), S_dev, L.S.bytes(), cudaMemcpyDeviceToDevice));
            built_ = false;  // the root's interface inverse is built again with it
            return;
        }
    throw Error(1, "no external child " + std::to_string(k));
}

void Composite::part_schur(int face, double* S_dev, cudaStream_t s)
{
    ensure_built();
    const int     r = tree_.root;
    const Domain& R = dom_[r];
    if (face < 0 || face > 3 || R.bc[face] != BC_ADJACENTED)
        throw Error(1, "the part's face toward its parent must be an Adjacented face of its root");
    for (const auto& k : tree_.children[r])
        if (k.first == face) throw Error(1, "the part's face toward its parent is connected inside the part");
    Link L;
    L.child = r;
    L.loc   = face ^ 1;  // the parent's face toward this part
    L.cn    = edge_length(face, R.nx, R.ny);
    link_schur(L, s);
    FPB_CUDA(cudaMemcpyAsync(S_dev, L.S.get(), L.S.bytes(), cudaMemcpyDeviceToDevice, s));
    FPB_CUDA(cudaStreamSynchronize(s));
}

void Composite::part_upward(double* const* fields, const double* const* ghosts, int face, double* edge_out,
                            cudaStream_t s, GmresInfo* info)
{
    ensure_built();
    mixed_ = false;
    assemble(fields, ghosts, s);
    auto bond = [&](double* dst, int dd, int loc, const double* src, int sd) {
        const Domain &A = dom_[dd], &B = dom_[sd];
        k_bond_add<double><<<grid_for(edge_length(loc, A.nx, A.ny), 128), 128, 0, s>>>(dst, A.nx, A.ny, loc, -1.0, src,
                                                                                     B.nx, B.ny);
        FPB_CHECK_LAUNCH();
    };
    const auto& T = tree_;
    for (int l = (int)T.levels.size() - 1; l >= 1; --l)
    {
        for (int d : T.levels[l])
        {
            double* td = temp_[d].as<double>();
            FPB_CUDA(cudaMemcpyAsync(td, fields[d], dom_[d].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
            for (auto& c : T.children[d])
            {
                bond(td, d, c.first, temp_[c.second].as<double>(), c.second);
                bond(fields[d], d, c.first, temp_[c.second].as<double>(), c.second);
            }
        }
        for (int d : T.levels[l]) node_solve(d, temp_[d].as<double>(), s, nullptr);
    }
    // the part's root is a non-root domain of the undivided tree: its solved copy goes to the parent
    const int r = T.root;
    if (!temp_[r].get()) temp_[r].alloc(dom_[r].cells() * sizeof(double));
    double* tr = temp_[r].as<double>();
    FPB_CUDA(cudaMemcpyAsync(tr, fields[r], dom_[r].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
    for (auto& c : T.children[r])
    {
        bond(tr, r, c.first, temp_[c.second].as<double>(), c.second);
        bond(fields[r], r, c.first, temp_[c.second].as<double>(), c.second);
    }
    node_solve(r, tr, s, info);
    const Domain& R = dom_[r];
    k_edge_gather<double><<<grid_for(edge_length(face, R.nx, R.ny), 128), 128, 0, s>>>(edge_out, tr, R.nx, R.ny, face);
    FPB_CHECK_LAUNCH();
}

void Composite::part_downward(double* const* fields, int face, const double* parent_edge, cudaStream_t s,
                              GmresInfo* info)
{
    const auto& T = tree_;
    const int   r = T.root;
    edge_axpy(fields[r], r, face, -1.0, parent_edge, s);
    node_solve(r, fields[r], s, info);
    for (size_t l = 1; l < T.levels.size(); ++l)
    {
        for (int d : T.levels[l])
        {
            const Domain &A = dom_[d], &B = dom_[T.parent[d].second];
            k_bond_add<double><<<grid_for(edge_length(T.parent[d].first, A.nx, A.ny), 128), 128, 0, s>>>(
                fields[d], A.nx, A.ny, T.parent[d].first, -1.0, fields[T.parent[d].second], B.nx, B.ny);
            FPB_CHECK_LAUNCH();
        }
        for (int d : T.levels[l]) node_solve(d, fields[d], s, nullptr);
    }
}

void Composite::root_solve(double* const* fields, const double* const* ghosts, const double* const* child_edges,
                           double* const* edges_out, cudaStream_t s, GmresInfo* info)
{
    mixed_ = false;
    assemble(fields, ghosts, s);
    eliminate(fields, s, info, child_edges, edges_out);
}

}  // namespace fpb
