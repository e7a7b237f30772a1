// C ABI (include/fp_capi.h fp_composite3d_*): ConcatPoissonSolver3D (pe/concat/concat_solver3d.cpp:5-247) on
// the device, for a tree of 3D boxes connected on whole faces.
//
// The algorithm is the reference's: boundary assembly from the six ghost planes per box (:159-247), scaling
// by hx^2, a bottom-up pass (copies of the subtrees' fields, each reduced by its children's solved copies and
// solved), the root equation, and a top-down pass (:100-157). A box with children is solved by GMRES on full
// 3D fields for (I - A^-1 S) x = A^-1 b (gmres_solver3d.cpp:155-306: modified Gram-Schmidt, Givens rotations,
// absolute tolerance on ||r|| at every restart and on |g_{j+1}| inside), with one dense Schur matrix per child
// (schur_mat3d.cpp): column c is the child's layer facing the parent after a solve of a unit impulse at cell c
// of that layer. The rectangle solves are DevRect3D (fp_rect3d.cu); the Schur columns of a leaf child come
// from batched impulse solves, chunked to bound memory.
//
// Layout: value(i, j, k) = f[(i ny + j) nz + k]. A face plane is indexed as the reference's Schur matrices
// index it: x faces (j, k), y faces (i, k), z faces (i, j), row-major.
#include "../../include/fp_capi.h"
#include "fp_composite.h"
#include "fp_gmres.cuh"
#include "fp_internal.h"
#include "fp_ops.cuh"
#include "fp_rect3d.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <vector>

namespace fpb
{
namespace
{
inline unsigned grid3(long long n, int block, int cap = 4096)
{
    const long long g = (n + block - 1) / block;
    return (unsigned)std::max(1LL, std::min<long long>(g, cap));
}

struct Box
{
    int       nx = 0, ny = 0, nz = 0;
    double    hx = 0, hy = 0, hz = 0;
    int       bc[6]{};
    long long cells() const { return (long long)nx * ny * nz; }
};

// The cells of one face layer of an (nx, ny, nz) field: cell (p, q) of the plane is f[base + p sp + q sq].
struct Plane
{
    long long base = 0, sp = 0, sq = 0;
    int       np = 0, nq = 0;
    long long size() const { return (long long)np * nq; }
};

Plane plane_of(const Box& b, int face)
{
    const long long nyz = (long long)b.ny * b.nz;
    const bool      hi  = face & 1;
    switch (face >> 1)
    {
        case 0: return Plane{(hi ? b.nx - 1 : 0) * nyz, b.nz, 1, b.ny, b.nz};
        case 1: return Plane{(long long)(hi ? b.ny - 1 : 0) * b.nz, nyz, 1, b.nx, b.nz};
        default: return Plane{hi ? b.nz - 1 : 0, nyz, b.nz, b.nx, b.ny};
    }
}

Plane flat_plane(const Plane& p) { return Plane{0, p.nq, 1, p.np, p.nq}; }

// dst's cells of plane pd += a * src's cells of plane ps (same np x nq)
__global__ void k3_plane_add(double* __restrict__ dst, const Plane pd, double a, const double* __restrict__ src,
                             const Plane ps)
{
    const long long n = (long long)pd.np * pd.nq;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    {
        const long long p = t / pd.nq, q = t - p * pd.nq;
        dst[pd.base + p * pd.sp + q * pd.sq] += a * src[ps.base + p * ps.sp + q * ps.sq];
    }
}

// out[t] = f's plane cell t (row-major)
__global__ void k3_plane_gather(double* __restrict__ out, const double* __restrict__ f, const Plane pf)
{
    const long long n = (long long)pf.np * pf.nq;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    {
        const long long p = t / pf.nq, q = t - p * pf.nq;
        out[t] = f[pf.base + p * pf.sp + q * pf.sq];
    }
}

// nb fields of `cells` values: field b = unit impulse at plane cell c0 + b (the fields are zero on entry)
__global__ void k3_impulses(double* fields, long long cells, const Plane pf, long long c0, int nb)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const long long c = c0 + b, p = c / pf.nq, q = c - p * pf.nq;
    fields[(long long)b * cells + pf.base + p * pf.sp + q * pf.sq] = 1.0;
}

// S[row, c0 + b] = field b's plane cell row, for nb solved impulse fields (S row-major cn x cn)
__global__ void k3_impulse_extract(const double* __restrict__ fields, long long cells, const Plane pf,
                                   double* __restrict__ S, long long cn, long long c0, int nb)
{
    const long long n = cn * nb;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x)
    {
        const long long b = t / cn, row = t - b * cn, p = row / pf.nq, q = row - p * pf.nq;
        S[row * cn + c0 + b] = fields[b * cells + pf.base + p * pf.sp + q * pf.sq];
    }
}

constexpr int  kFaces = 6;
constexpr long kImpulseBytes = 256L << 20;  // device memory for one chunk of batched impulse solves

struct Child3
{
    int    face = 0;  // face of the parent
    int    child = 0;
    Plane  pp;        // the parent's layer at `face`
    long long cn = 0;
    DevBuf S;         // cn x cn, row-major
};

struct Node3
{
    std::vector<Child3> kids;
    DevBuf              V, w, r, x, ft, vec, prod;  // GMRES on full fields ((m + 1) x cells for V)
    DevBuf              hd;                         // H column, residual norm, y (m + 2 doubles)
    DevBuf              b, vin;                     // the solve's A^-1 b and the Arnoldi step's input
    DevBuf              arr, st;                    // GmArrays storage, GmState
    cudaGraphExec_t     graph = nullptr;            // the GMRES loop (built on first use per parameters)
    ~Node3()
    {
        if (graph) cudaGraphExecDestroy(graph);
    }
    Node3() = default;
    Node3(Node3&& o) noexcept
        : kids(std::move(o.kids)), V(std::move(o.V)), w(std::move(o.w)), r(std::move(o.r)), x(std::move(o.x)),
          ft(std::move(o.ft)), vec(std::move(o.vec)), prod(std::move(o.prod)), hd(std::move(o.hd)), b(std::move(o.b)),
          vin(std::move(o.vin)), arr(std::move(o.arr)), st(std::move(o.st)), graph(o.graph)
    {
        o.graph = nullptr;
    }
};

}  // namespace

class Composite3D
{
public:
    Composite3D(const std::vector<Box>& boxes, const std::vector<std::array<int, 3>>& conns, int root, int m,
                double tol, int max_iter)
        : box_(boxes), m_(m), tol_(tol), max_iter_(max_iter)
    {
        const int nd = (int)box_.size();
        tree_        = build_tree(nd, conns, root, kFaces);
        for (const auto& c : conns)
        {
            const int a = c[0], f = c[1], b = c[2];
            const Plane pa = plane_of(box_[a], f), pb = plane_of(box_[b], f ^ 1);
            if (pa.np != pb.np || pa.nq != pb.nq)
                throw Error(FP_ERR_INVALID, "connected faces of domains " + std::to_string(a) + " and " +
                                                std::to_string(b) + " have different cell counts");
            box_[a].bc[f]     = BC_ADJACENTED;
            box_[b].bc[f ^ 1] = BC_ADJACENTED;
        }
        rect_.resize(nd);
        for (int d = 0; d < nd; ++d)
        {
            const Box& B = box_[d];
            rect_[d].reset(new DevRect3D(B.nx, B.ny, B.nz, B.hx, B.hy, B.hz, B.bc));
        }
        node_.resize(nd);
        temp_.resize(nd);
        for (int d = 0; d < nd; ++d)
        {
            if (d != tree_.root) temp_[d].alloc(box_[d].cells() * sizeof(double));
            for (const auto& kc : tree_.children[d])
            {
                Child3 k;
                k.face  = kc.first;
                k.child = kc.second;
                k.pp    = plane_of(box_[d], k.face);
                k.cn    = k.pp.size();
                node_[d].kids.push_back(std::move(k));
            }
        }
        red_.alloc((kRedBlocks + 8) * sizeof(double));
        FPB_CUDA(cudaMemset(red_.get(), 0, red_.bytes()));
        FPB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&gmst_), sizeof(GmState)));
        set_parameter(m, tol, max_iter);
    }
    ~Composite3D()
    {
        if (gmst_) cudaFreeHost(gmst_);
    }

    // ConcatPoissonSolver3D::set_parameter (concat_solver3d.cpp:5-18): the Schur matrices are built again
    // (they depend on the GMRES parameters through the impulse solves of children that have children).
    void set_parameter(int m, double tol, int max_iter)
    {
        if (m < 1 || m > kMaxM) throw Error(FP_ERR_INVALID, "m must be in [1, " + std::to_string(kMaxM) + "]");
        if (!(tol > 0) || max_iter < 1) throw Error(FP_ERR_INVALID, "tol must be > 0 and max_iter >= 1");
        const bool changed = m != m_ || tol != tol_ || max_iter != max_iter_ || !built_;
        m_        = m;
        tol_      = tol;
        max_iter_ = max_iter;
        if (!changed) return;
        for (int d = 0; d < (int)box_.size(); ++d)
        {
            Node3& N = node_[d];
            if (N.kids.empty()) continue;
            const size_t cells = (size_t)box_[d].cells();
            N.V.ensure((size_t)(m_ + 1) * cells * sizeof(double));
            for (DevBuf* b : {&N.w, &N.r, &N.x, &N.ft}) b->ensure(cells * sizeof(double));
            long long cmax = 0;
            for (const auto& k : N.kids) cmax = std::max(cmax, k.cn);
            N.vec.ensure((size_t)cmax * sizeof(double));
            N.prod.ensure((size_t)cmax * sizeof(double));
            N.hd.ensure((size_t)(m_ + 2) * sizeof(double));
            for (DevBuf* b : {&N.b, &N.vin}) b->ensure(cells * sizeof(double));
            N.arr.ensure((size_t)((m_ + 1) * m_ + 3 * m_ + 1) * sizeof(double));
            N.st.ensure(sizeof(GmState));
            if (N.graph) cudaGraphExecDestroy(N.graph);
            N.graph = nullptr;
        }
        build_schur();
        built_ = true;
    }

    const Tree& tree() const { return tree_; }
    const std::vector<Box>& boxes() const { return box_; }

    // ConcatPoissonSolver3D::solve on device fields (in place); ghosts: 6 device pointers per box or null.
    void solve(double* const* f, const double* const* ghosts, cudaStream_t s, GmresInfo* info)
    {
        const int nd = (int)box_.size();
        assemble(f, ghosts, s);
        for (int d = 0; d < nd; ++d)
        {
            const double a = box_[d].hx * box_[d].hx;
            k_scale<<<grid3(box_[d].cells(), 256), 256, 0, s>>>(f[d], a, box_[d].cells());
            FPB_CHECK_LAUNCH();
        }
        const auto& L = tree_.levels;
        for (int l = (int)L.size() - 1; l >= 1; --l)
        {
            for (int d : L[l])
            {
                double* t = temp_[d].as<double>();
                FPB_CUDA(cudaMemcpyAsync(t, f[d], box_[d].cells() * sizeof(double), cudaMemcpyDeviceToDevice, s));
                for (const auto& k : node_[d].kids)
                {
                    bond_add(t, d, k.face, temp_[k.child].as<double>(), k.child, s);
                    bond_add(f[d], d, k.face, temp_[k.child].as<double>(), k.child, s);
                }
            }
            for (int d : L[l]) node_solve(d, temp_[d].as<double>(), s, nullptr);
        }
        const int r = tree_.root;
        for (const auto& k : node_[r].kids) bond_add(f[r], r, k.face, temp_[k.child].as<double>(), k.child, s);
        node_solve(r, f[r], s, info);
        for (int l = 1; l < (int)L.size(); ++l)
        {
            for (int d : L[l])
            {
                const auto& pr = tree_.parent[d];
                bond_add(f[d], d, pr.first, f[pr.second], pr.second, s);
            }
            for (int d : L[l]) node_solve(d, f[d], s, nullptr);
        }
    }

private:
    static constexpr int kMaxM = 512;

    // field3::bond_add(face, -1, neighbour) (field3.cpp:306-375): dst's layer at `face` -= the neighbour's layer
    // on the opposite face
    void bond_add(double* dst, int d, int face, const double* nb, int n, cudaStream_t s)
    {
        const Plane pd = plane_of(box_[d], face), ps = plane_of(box_[n], face ^ 1);
        k3_plane_add<<<grid3(pd.size(), 256), 256, 0, s>>>(dst, pd, -1.0, nb, ps);
        FPB_CHECK_LAUNCH();
    }

    // concat_solver3d.cpp:159-247: Dirichlet ghost planes enter with -1/h^2, then Neumann ones with +-1/h
    void assemble(double* const* f, const double* const* ghosts, cudaStream_t s)
    {
        if (!ghosts) return;
        for (int d = 0; d < (int)box_.size(); ++d)
        {
            const Box&   B     = box_[d];
            const double hs[6] = {B.hx, B.hx, B.hy, B.hy, B.hz, B.hz};
            for (int pass = 0; pass < 2; ++pass)
                for (int face = 0; face < kFaces; ++face)
                {
                    const double* g = ghosts[kFaces * d + face];
                    if (!g) continue;
                    double a;
                    if (pass == 0 && B.bc[face] == BC_DIRICHLET) a = -1.0 / hs[face] / hs[face];
                    else if (pass == 1 && B.bc[face] == BC_NEUMANN) a = ((face & 1) ? -1.0 : 1.0) / hs[face];
                    else continue;
                    const Plane pf = plane_of(B, face);
                    k3_plane_add<<<grid3(pf.size(), 256), 256, 0, s>>>(f[d], pf, a, g, flat_plane(pf));
                    FPB_CHECK_LAUNCH();
                }
        }
    }

    // solver_map[d]->solve: PoissonSolver3D for a leaf, GMRESSolver3D for a box with children
    void node_solve(int d, double* f, cudaStream_t s, GmresInfo* info)
    {
        if (node_[d].kids.empty()) rect_[d]->solve(f, 1, s);
        else gmres(d, f, s, info);
    }

    void node_solve_batch(int d, double* f, long long batch, cudaStream_t s)
    {
        if (node_[d].kids.empty())
        {
            rect_[d]->solve(f, batch, s);
            return;
        }
        for (long long b = 0; b < batch; ++b) gmres(d, f + b * box_[d].cells(), s, nullptr);
    }

    // SchurMat3D_*::construct for every child of every box, deepest boxes first (the impulse solves of a child
    // that has children run its own GMRES, whose matrices are then ready)
    void build_schur()
    {
        const auto& L = tree_.levels;
        cudaStream_t s = 0;
        for (int l = (int)L.size() - 1; l >= 0; --l)
            for (int d : L[l])
                for (auto& k : node_[d].kids)
                {
                    const Box&      C     = box_[k.child];
                    const Plane     pc    = plane_of(C, k.face ^ 1);
                    const long long cells = C.cells();
                    const long long chunk =
                        std::max<long long>(1, std::min<long long>(k.cn, kImpulseBytes / (cells * (long long)sizeof(double))));
                    k.S.ensure((size_t)(k.cn * k.cn) * sizeof(double));
                    DevBuf buf((size_t)(chunk * cells) * sizeof(double));
                    for (long long c0 = 0; c0 < k.cn; c0 += chunk)
                    {
                        const int nb = (int)std::min<long long>(chunk, k.cn - c0);
                        FPB_CUDA(cudaMemsetAsync(buf.get(), 0, (size_t)(nb * cells) * sizeof(double), s));
                        k3_impulses<<<grid3(nb, 128), 128, 0, s>>>(buf.as<double>(), cells, pc, c0, nb);
                        FPB_CHECK_LAUNCH();
                        node_solve_batch(k.child, buf.as<double>(), nb, s);
                        k3_impulse_extract<<<grid3(k.cn * nb, 256), 256, 0, s>>>(buf.as<double>(), cells, pc,
                                                                                 k.S.as<double>(), k.cn, c0, nb);
                        FPB_CHECK_LAUNCH();
                    }
                }
        FPB_CUDA(cudaDeviceSynchronize());
    }

    // out = in - A^-1 sum_k S_k in (GMRESSolver3D::Afun, gmres_solver3d.cpp:122-136)
    void afun(int d, const double* in, double* out, cudaStream_t s)
    {
        Node3&          N     = node_[d];
        const long long cells = box_[d].cells();
        double*         ft    = N.ft.as<double>();
        FPB_CUDA(cudaMemsetAsync(ft, 0, cells * sizeof(double), s));
        for (const auto& k : N.kids)
        {
            k3_plane_gather<<<grid3(k.cn, 256), 256, 0, s>>>(N.vec.as<double>(), in, k.pp);
            FPB_CHECK_LAUNCH();
            const int warps = 8;
            k_dense_matvec<<<(unsigned)((k.cn + warps - 1) / warps), warps * 32, 0, s>>>(
                k.S.as<double>(), (int)k.cn, N.vec.as<double>(), N.prod.as<double>(), 0);
            FPB_CHECK_LAUNCH();
            k3_plane_add<<<grid3(k.cn, 256), 256, 0, s>>>(ft, k.pp, 1.0, N.prod.as<double>(), flat_plane(k.pp));
            FPB_CHECK_LAUNCH();
        }
        rect_[d]->solve(ft, 1, s);
        k_sub<<<grid3(cells, 256), 256, 0, s>>>(out, in, ft, cells);
        FPB_CHECK_LAUNCH();
    }

    // dev_out = a . b (sqrt of it with take_sqrt), on the device
    void dot(const double* a, const double* b, long long n, bool take_sqrt, double* dev_out, cudaStream_t s)
    {
        double*   partials = red_.as<double>();
        unsigned* ticket   = reinterpret_cast<unsigned*>(partials + kRedBlocks);
        k_dot<<<grid3(n, kRedThreads, kRedBlocks), kRedThreads, 0, s>>>(a, b, n, partials, ticket, dev_out,
                                                                         take_sqrt ? 1 : 0);
        FPB_CHECK_LAUNCH();
    }

    GmArrays arrays(int d)
    {
        Node3&   N = node_[d];
        double*  p = N.arr.as<double>();
        GmArrays a;
        a.H    = p;
        a.cs   = a.H + (size_t)(m_ + 1) * m_;
        a.sn   = a.cs + m_;
        a.g    = a.sn + m_;
        a.y    = a.g + (m_ + 1);
        a.hcol = N.hd.as<double>();
        return a;
    }

    // The GMRES loop of box d as one graph (fp_gmres.cuh) on the node's fixed buffers (b, x, V, w, r, vin).
    void build_gmres_graph(int d, cudaStream_t s)
    {
        Node3&          N = node_[d];
        const long long n = box_[d].cells();
        GmBuffers       B;
        B.V        = N.V.as<double>();
        B.w        = N.w.as<double>();
        B.r        = N.r.as<double>();
        B.x        = N.x.as<double>();
        B.b        = N.b.as<double>();
        B.vin      = N.vin.as<double>();
        B.st       = N.st.as<GmState>();
        B.a        = arrays(d);
        B.partials = red_.as<double>();
        B.ticket   = reinterpret_cast<unsigned*>(B.partials + kRedBlocks);
        // warm-up outside the capture: the rectangle solve's work buffers are allocated on first use
        afun(d, B.x, B.w, s);
        FPB_CUDA(cudaStreamSynchronize(s));
        N.graph = capture_gmres(
            n, m_, tol_, max_iter_, false, B, [&](const double* in, double* out, cudaStream_t q) { afun(d, in, out, q); },
            [](cudaStream_t) {},
            [&](const double* x, const double* y, long long len, bool sq, double* out, cudaStream_t q) {
                dot(x, y, len, sq, out, q);
            });
    }

    // GMRESSolver3D::solve (gmres_solver3d.cpp:155-306) on the full field f, in place: A^-1 f and the copies into
    // the node's buffers on the stream, then the loop as one graph launch, one wait for its state
    void gmres(int d, double* f, cudaStream_t s, GmresInfo* info)
    {
        Node3&          N = node_[d];
        const long long n = box_[d].cells();
        rect_[d]->solve(f, 1, s);  // b <- A^-1 b
        FPB_CUDA(cudaMemcpyAsync(N.b.get(), f, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        FPB_CUDA(cudaMemcpyAsync(N.x.get(), f, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        if (!N.graph) build_gmres_graph(d, s);
        FPB_CUDA(cudaGraphLaunch(N.graph, s));
        FPB_CUDA(cudaMemcpyAsync(f, N.x.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        FPB_CUDA(cudaMemcpyAsync(gmst_, N.st.get(), sizeof(GmState), cudaMemcpyDeviceToHost, s));
        FPB_CUDA(cudaStreamSynchronize(s));
        const GmState st = *gmst_;
        if (st.err) throw Error(FP_ERR_NAN, "non-finite GMRES value");
        if (info)
        {
            info->iterations += st.iters;
            info->restarts += st.restarts;
            info->residual  = st.beta;
            info->converged = info->converged && st.converged;
        }
    }

    std::vector<Box>                        box_;
    Tree                                    tree_;
    std::vector<std::unique_ptr<DevRect3D>> rect_;
    std::vector<Node3>                      node_;
    std::vector<DevBuf>                     temp_;
    DevBuf                                  red_;
    GmState*                                gmst_  = nullptr;  // pinned copy of a GMRES run's state
    int                                     m_     = 0;
    double                                  tol_   = 0;
    int                                     max_iter_ = 0;
    bool                                    built_ = false;
};

}  // namespace fpb

struct fp_composite3d
{
    std::unique_ptr<fpb::Composite3D> c;
    std::vector<fpb::DevBuf>          fields, ghosts;
};

using namespace fpb;

extern "C" {

int fp_composite3d_create(const fp_geometry3* g, int m, double tol, int max_iter, fp_composite3d** out)
{
    return guarded([&] {
        if (!out) throw Error(FP_ERR_INVALID, "null output handle");
        *out = nullptr;
        if (!g || g->n_domains <= 0 || !g->nx || !g->ny || !g->nz || !g->hx || !g->hy || !g->hz || !g->bc)
            throw Error(FP_ERR_INVALID, "incomplete geometry description");
        if (g->n_connections > 0 && !g->connections) throw Error(FP_ERR_INVALID, "null connection list");
        require_device();
        std::vector<Box> boxes(g->n_domains);
        for (int d = 0; d < g->n_domains; ++d)
        {
            Box& B = boxes[d];
            B.nx   = g->nx[d];
            B.ny   = g->ny[d];
            B.nz   = g->nz[d];
            B.hx   = g->hx[d];
            B.hy   = g->hy[d];
            B.hz   = g->hz[d];
            for (int f = 0; f < 6; ++f) B.bc[f] = g->bc[6 * d + f];
        }
        std::vector<std::array<int, 3>> conns(g->n_connections);
        for (int k = 0; k < g->n_connections; ++k)
            conns[k] = {g->connections[3 * k], g->connections[3 * k + 1], g->connections[3 * k + 2]};
        std::unique_ptr<fp_composite3d> h(new fp_composite3d());
        h->c.reset(new Composite3D(boxes, conns, g->root, m, tol, max_iter));
        *out = h.release();
    });
}

int fp_composite3d_set_parameter(fp_composite3d* c, int m, double tol, int max_iter)
{
    return guarded([&] {
        if (!c) throw Error(FP_ERR_INVALID, "null solver");
        c->c->set_parameter(m, tol, max_iter);
    });
}

int fp_composite3d_solve_f64(fp_composite3d* c, double* const* fields, const double* const* ghosts, int flags,
                             void* stream, fp_solve_info* info)
{
    GmresInfo gi;
    int       rc = guarded([&] {
        if (!c) throw Error(FP_ERR_INVALID, "null solver");
        if (!fields) throw Error(FP_ERR_INVALID, "null field list");
        const auto& boxes = c->c->boxes();
        const int   nd    = (int)boxes.size();
        for (int d = 0; d < nd; ++d)
            if (!fields[d]) throw Error(FP_ERR_INVALID, "null field pointer");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (flags & FP_DEVICE)
        {
            c->c->solve(fields, ghosts, s, &gi);
            if (flags & FP_SYNC) FPB_CUDA(cudaStreamSynchronize(s));
        }
        else
        {
            c->fields.resize(nd);
            c->ghosts.resize(6 * nd);
            std::vector<double*>       dev(nd);
            std::vector<const double*> gdev(6 * nd, nullptr);
            for (int d = 0; d < nd; ++d)
            {
                const size_t bytes = (size_t)boxes[d].cells() * sizeof(double);
                c->fields[d].ensure(bytes);
                dev[d] = c->fields[d].as<double>();
                FPB_CUDA(cudaMemcpyAsync(dev[d], fields[d], bytes, cudaMemcpyHostToDevice, s));
                for (int f = 0; f < 6 && ghosts; ++f)
                {
                    if (!ghosts[6 * d + f]) continue;
                    const Plane  p  = plane_of(boxes[d], f);
                    const size_t gb = (size_t)p.size() * sizeof(double);
                    c->ghosts[6 * d + f].ensure(gb);
                    FPB_CUDA(cudaMemcpyAsync(c->ghosts[6 * d + f].get(), ghosts[6 * d + f], gb, cudaMemcpyHostToDevice, s));
                    gdev[6 * d + f] = c->ghosts[6 * d + f].as<double>();
                }
            }
            c->c->solve(dev.data(), ghosts ? gdev.data() : nullptr, s, &gi);
            for (int d = 0; d < nd; ++d)
                FPB_CUDA(cudaMemcpyAsync(fields[d], dev[d], (size_t)boxes[d].cells() * sizeof(double),
                                         cudaMemcpyDeviceToHost, s));
            FPB_CUDA(cudaStreamSynchronize(s));
        }
        if ((flags & FP_CHECK_CONVERGENCE) && !gi.converged)
            throw Error(FP_ERR_NOT_CONVERGED, "GMRES stopped at max_iter above tol (residual " +
                                                  std::to_string(gi.residual) + ")");
    });
    if (info)
    {
        info->gmres_iterations = gi.iterations;
        info->gmres_restarts   = gi.restarts;
        info->gmres_residual   = gi.residual;
        info->converged        = gi.converged ? 1 : 0;
        info->refinements      = 0;
        info->rel_change       = 0.0;
    }
    return rc;
}

int fp_composite3d_tree(const fp_composite3d* c, int* root, int* level_of)
{
    return guarded([&] {
        if (!c || !root || !level_of) throw Error(FP_ERR_INVALID, "null argument");
        const Tree& t = c->c->tree();
        *root         = t.root;
        for (size_t l = 0; l < t.levels.size(); ++l)
            for (int d : t.levels[l]) level_of[d] = (int)l;
    });
}

int fp_composite3d_destroy(fp_composite3d* c)
{
    return guarded([&] { delete c; });
}

}  // extern "C"
