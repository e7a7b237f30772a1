// Batched composite solves: many independent ConcatPoissonSolver2D problems of uneven sizes solved in
// lockstep, every stage one launch over all problems (heterogeneous work lists, persistent kernels).
//
// Scope: each problem is a root rectangle with Dirichlet faces and leaf rectangles attached on full faces
// (a depth-1 tree: the L / T / cross shapes), each leaf's sides along its interface Dirichlet, its far
// face Dirichlet or Neumann, and nx of every subdomain a multiple of 32 (>= 64). The root operator is
// then diagonalised by DST-I in both directions and every leaf shares the root's basis along its
// interface, so the interface operator I - P A^-1 S of the reference's Schur GMRES
// (pe/concat/gmres_solver2d.cpp:90-104) is known in closed form: diagonal in the y-DST basis on the
// root's x faces (leaf responses by continued fractions, Neumann ends included), diagonal in the x-DST
// basis on its y faces (leaf responses from the leaf's own y family, DD / ND / DN), plus a dense cross
// block. The batch solves it exactly (a small reduced system per problem, its inverse built at
// creation), which is the solution the reference's GMRES converges to.
#pragma once

#include "fp_composite.h"

#include <array>
#include <memory>
#include <vector>

namespace fpb
{

struct BatchProblemDesc
{
    std::vector<Domain>             doms;   // bc with Adjacented on connected faces
    std::vector<std::array<int, 3>> conns;  // (a, face of a, b)
};

struct BatchTiming  // autotuned launch shapes
{
    int dst_threads = 256, dst_blocks_per_sm = 2, chase_threads = 256;
};

class BatchBase
{
public:
    virtual ~BatchBase() {}
    // fields: one device pointer per subdomain, problems back to back in the order given at creation.
    // ghosts: 4 per subdomain (device, may be null) or null. steps == 0: one solve in the storage
    // precision; steps >= 1: that many inner solves in FP64 iterative refinement (residual of the
    // composite operator in FP64).
    virtual void solve(double* const* fields, const double* const* ghosts, int steps, cudaStream_t s) = 0;
    // The same launch sequence captured once into a CUDA graph (per field pointers and steps) and replayed.
    virtual void solve_graph(double* const* fields, const double* const* ghosts, int steps, cudaStream_t s) = 0;
    virtual long long graph_kernels() const = 0;  // kernels in the captured graph
    // Iterative refinement until |correction| <= rel_tol |u| over all cells (or the observed contraction
    // predicts it after the last correction), at most max_refine inner solves. Returns the steps taken;
    // *rel_change the last |correction| / |u|.
    // first: when given, the first inner solve runs on that solver (same problems; e.g. the FP64 solve
    // followed by FP32 corrections).
    // With max_refine > 1 the whole refinement is one CUDA graph (captured once per field pointers, first
    // solver and parameters) whose loop over the corrections is a conditional while node: a device kernel
    // applies the stop rule after every correction, so the host waits once, for the result. With
    // max_refine == 1 the loop runs on the host. defer: queue the work and return -1 without waiting;
    // refine_result then gives the outcome once the stream has completed.
    virtual int refine(double* const* fields, const double* const* ghosts, double rel_tol, int max_refine,
                       cudaStream_t s, double* rel_change, BatchBase* first = nullptr, bool defer = false) = 0;
    // Outcome of the deferred refinements queued since the last call (the stream must have completed):
    // steps and change of the last one. Throws if any of them met a non-finite value.
    virtual void refine_result(int* steps, double* rel_change) = 0;
    // One inner solve of already assembled, hx^2-scaled right-hand sides `in` (one pointer per subdomain)
    // into `out` (stored, not accumulated); in and out may alias.
    virtual void solve_assembled(const double* const* in, double* const* out, cudaStream_t s) = 0;
    // The work lists solve_assembled(in, out, .) uses, built now (outside any stream capture); the
    // generation counts how often they were rebuilt.
    virtual void      prepare_assembled(const double* const* in, double* const* out) = 0;
    virtual long long assembled_generation() const = 0;
    // Per-problem |fs - A u| / |fs| (fs: assembled, hx^2-scaled right-hand side); out: host, n_problems.
    virtual void residuals(const double* const* u, const double* const* rhs, const double* const* ghosts,
                           cudaStream_t s, double* out) = 0;
    virtual int  n_problems() const = 0;
    virtual int  n_domains() const  = 0;
    virtual const Domain& domain(int g) const = 0;
    virtual BatchTiming   timing() const      = 0;
    virtual void          autotune(cudaStream_t s) = 0;
};

// precision: 0 = FP64 storage and arithmetic, 1 = FP32 storage and arithmetic in the inner solves.
std::unique_ptr<BatchBase> make_batch(const std::vector<BatchProblemDesc>& probs, int precision);

}  // namespace fpb
