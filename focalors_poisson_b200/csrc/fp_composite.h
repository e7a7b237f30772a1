// Composite-geometry solver: the reference's ConcatPoissonSolver2D (pe/concat/concat_solver2d.cpp)
// with its Schur-complement GMRES (pe/concat/gmres_solver2d.cpp) on the GPU.
#pragma once

#include "fp_internal.h"

#include <array>
#include <memory>
#include <vector>

namespace fpb
{

struct Domain
{
    int    nx = 0, ny = 0;
    double hx = 0, hy = 0;
    int    bc[4]{};  // with Adjacented on connected faces
    long long cells() const { return (long long)nx * ny; }
};

struct GmState;  // fp_gmres.cuh

struct Tree
{
    int                                   root = 0;
    std::vector<std::vector<std::pair<int, int>>> children;  // d -> [(face of d, child)]
    std::vector<std::pair<int, int>>      parent;            // d -> (face of d toward its parent, parent)
    std::vector<std::vector<int>>         levels;            // BFS levels, root first
};

// Geometry2D::build_tree (base/domain/geometry2d.cpp:165-176) over TreeUtils
// (base/domain/geometry_tree.hpp:22-200). The root is the tree centre found by leaf stripping; a tie
// between two centres goes to the lower domain index (the reference compares addresses). Children are
// listed in face order. Throws on a disconnected or cyclic geometry. faces: 4 (2D, x-, x+, y-, y+) or 6
// (Geometry3D::build_tree, base/domain/geometry3d.cpp:151-160, adds z-, z+).
Tree build_tree(int nd, const std::vector<std::array<int, 3>>& conns, int root, int faces = 4);

struct GmresInfo
{
    int    iterations = 0;  // Arnoldi steps over all solves of the root node
    int    restarts   = 0;
    double residual   = 0;  // last residual norm of the root GMRES
    bool   converged  = true;
};

enum GmresMode : int
{
    GMRES_INTERFACE = 0,  // Krylov vectors on the interface unknowns (default)
    GMRES_FULLFIELD = 1   // Krylov vectors are full fields, like the reference
};

class Composite
{
public:
    // interface_inverse: build the inverse of each node's dense interface operator I - P A^-1 S at
    // creation and use it to precondition the interface GMRES (interface mode, n_if <= kMaxInverse).
    // ext: children of the root that live in other parts of a subtree decomposition, as (root face, its
    // interface length); their Schur matrices arrive through set_external_schur before the first solve.
    Composite(const std::vector<Domain>& doms, const std::vector<std::array<int, 3>>& conns, int root, int m,
              double tol, int max_iter, int mode, bool interface_inverse = true,
              const std::vector<std::array<int, 2>>& ext = {});
    static constexpr int kMaxInverse = 16384;
    ~Composite();
    void set_parameter(int m, double tol, int max_iter);
    // fields[d]: device pointers (nx*ny doubles) solved in place; ghosts[4*d+face]: device or null.
    void solve(double* const* fields, const double* const* ghosts, cudaStream_t s, GmresInfo* info);
    // Same problem by iterative refinement: inner solves with FP32 transforms (FP64 chase, FP64
    // interface operations, the interface inverse applied once without the residual test), FP64
    // residual of the composite operator, until |correction| <= rel_tol |u| or max_refine steps.
    // Returns the number of refinement steps; *rel_change gets the last |correction| / |u|.
    int solve_ir(double* const* fields, const double* const* ghosts, cudaStream_t s, double rel_tol, int max_refine,
                 double* rel_change, GmresInfo* info, bool inner_fp32 = true);
    // Transposed solve (adjoint of fields -> solution, ghosts held fixed): g <- H A^-1 g in place, H =
    // diag(hx^2) per domain, A the composite operator (symmetric). FP_ERR_UNSUPPORTED without a Dirichlet face.
    void solve_adjoint(double* const* fields, cudaStream_t s, GmresInfo* info);
    // The same by iterative refinement (FP32 or FP64 inner solves, FP64 residual), as solve_ir.
    int solve_adjoint_ir(double* const* fields, cudaStream_t s, double rel_tol, int max_refine, double* rel_change,
                         GmresInfo* info, bool inner_fp32 = true);
    // fields *= hx^2 (by_h2) or /= hx^2, per domain
    void scale_fields(double* const* fields, bool by_h2, cudaStream_t s);
    void require_nonsingular() const;
    // |fs - A u| / |fs| over all cells, fs = the assembled, hx^2-scaled right-hand side of (rhs, ghosts).
    // rhs is not modified (a copy is assembled).
    double residual_norm(const double* const* u, const double* const* rhs, const double* const* ghosts, cudaStream_t s);

    const Tree&                tree() const { return tree_; }
    const std::vector<Domain>& domains() const { return dom_; }
    // Builds the Schur matrices and interface inverses now rather than on the first solve that needs them.
    void prepare() { ensure_built(); }

    // Subtree decomposition: the composite solve split into parts solved on different GPUs. The root part
    // holds the root domain with its children outside (ext at construction); a subtree part holds the subtree
    // of one child of the root, whose face toward the root is an Adjacented face of the part's geometry. The
    // parts exchange one interface vector each way per solve; the results equal the undivided solve's.
    //   part_schur:    the Schur matrix of this part's root toward its parent across `face` (a face of the
    //                  part's root), cn x cn on the device, as the undivided solver builds it
    //   part_upward:   assembly, hx^2 scaling and the upward pass including the part's root; edge_out gets
    //                  the solved copy's values along `face` (for the parent's right-hand side)
    //   part_downward: the part root's field loses parent_edge along `face`, then the root solve and the
    //                  downward pass
    //   root_solve:    assembly, scaling, child_edges[k] subtracted along external child k's face, the root
    //                  solve (GMRES with the external Schur matrices), edges_out[k] = the solution along face k
    void set_external_schur(int k, const double* S_dev);
    void part_schur(int face, double* S_dev, cudaStream_t s);
    void part_upward(double* const* fields, const double* const* ghosts, int face, double* edge_out, cudaStream_t s,
                     GmresInfo* info);
    void part_downward(double* const* fields, int face, const double* parent_edge, cudaStream_t s, GmresInfo* info);
    void root_solve(double* const* fields, const double* const* ghosts, const double* const* child_edges,
                    double* const* edges_out, cudaStream_t s, GmresInfo* info);
    int  external_children() const { return n_ext_; }

private:
    struct Link
    {
        int    child, loc, cn, off;
        DevBuf S;  // cn x cn, S[j*cn + i] = child response at interface cell j to an impulse at cell i
    };
    struct Node
    {
        std::vector<Link> kids;
        int               n_if = 0;
        long long         n    = 0;  // Krylov vector length
        DevBuf            V, w, r, x, b, R, hcol, tmp;
        DevBuf            X, Z;  // interface inverse (n_if x n_if) and A^-1 S y workspace
        DevBuf            vin, arr, st;  // device GMRES loop: step input, Hessenberg storage, state
        bool              has_inv = false;
    };

    void build_schur();
    void build_gmres_graph(int d, cudaStream_t s);
    void drop_gmres_graphs();
    void link_schur(Link& L, cudaStream_t s);
    bool schur_by_spectral(Link& L, cudaStream_t s);
    void edge_axpy(double* field, int d, int loc, double a, const double* v, cudaStream_t s);
    void ensure_built();
    bool built_ = false;
    void assemble(double* const* fields, const double* const* ghosts, cudaStream_t s);
    void eliminate(double* const* fields, cudaStream_t s, GmresInfo* info, const double* const* child_edges = nullptr,
                   double* const* edges_out = nullptr);
    void rect_solve(int d, double* f, long long batch, cudaStream_t s) const;
    void residual_into(double* const* r, const double* const* fs, const double* const* u, cudaStream_t s);
    void ensure_ir_workspace();
    int  refine(double* const* fields, cudaStream_t s, double rel_tol, int max_refine, double* rel_change,
                GmresInfo* info, bool inner_fp32);  // fields: assembled, scaled RHS in, solution out
    void scale_by_h2(double* const* fields, cudaStream_t s);
    void build_interface_inverse(int d);
    bool refine_with_inverse(int d, double* f, cudaStream_t s, GmresInfo* info);
    void node_solve(int d, double* f, cudaStream_t s, GmresInfo* info);
    void afun(int d, const double* v, double* out, cudaStream_t s);
    void schur_apply_into(int d, const double* vec, bool vec_is_field, double* R, cudaStream_t s);
    double dot(const double* a, const double* b, long long n, bool sqrt_, cudaStream_t s, double* dev_out);

    std::vector<Domain>                          dom_;
    Tree                                         tree_;
    int                                          m_, max_iter_, mode_;
    bool                                         want_inverse_ = true;
    double                                       tol_;
    std::vector<std::unique_ptr<DevRect<double>>> rect_;
    std::vector<Node>                            node_;
    std::vector<DevBuf>                          temp_;    // per non-root domain (upward sweep temporaries)
    std::vector<DevBuf>                          fs_, u_;  // iterative refinement: scaled RHS, solution
    DevBuf                                       sums_;    // per-domain reduction results
    bool                                         mixed_ = false;  // inner solve of iterative refinement
    DevBuf                                       red_;     // reduction scratch: partials + ticket + results
    int                                          n_ext_ = 0;  // external children of the root (subtree parts)
    std::vector<cudaGraphExec_t>                 gm_graph_;   // per node: the GMRES loop (fp_gmres.cuh)
    GmState*                                     gm_host_ = nullptr;  // pinned copy of a loop's outcome
};

}  // namespace fpb
