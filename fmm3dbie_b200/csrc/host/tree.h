// Cluster trees and the dual traversal of the hierarchical far field.
//
// The far field u(t) = sum_s [c_s G(t,s) + d_s n_s . grad_s G(t,s)] over all
// oversampled sources (the role of lfmm3d / hfmm3d at the call sites
// lap_comb_dir.f90:1094 and helm_comb_dir.f:1117) is evaluated with
// kernel-independent barycentric Lagrange interpolation on Chebyshev grids
// (a dual-tree treecode in the manner of Wang, Tlupova and Krasny, "A
// kernel-independent treecode based on barycentric Lagrange interpolation",
// Commun. Comput. Phys. 28 (2020), and its dual-traversal variant):
//
//  * a source cluster S with a proxy grid y_k carries proxy charges
//      q_k = sum_{s in S} [c_s L_k(s) + d_s n_s . grad L_k(s)],
//    so that sum_{s in S} [...] ~= sum_k q_k G(t, y_k) for targets t that
//    are well separated from S;
//  * a target cluster T with a proxy grid x_k receives proxy potentials
//    phi_k and passes them to its targets as u(t) += sum_k L_k(t) phi_k.
//
// Both trees are k-d trees: a node splits its points in two along the
// longest side of its tight bounding box, at a multiple of 32 points near the
// median, so that leaves hold between half and all of the leaf size and the
// target leaves fill whole warps of the thread block that evaluates them.
// The dual traversal
// accepts a pair (T, S) when r_T + r_S < theta |c_T - c_S| and then picks
// the cheapest of the four forms particle-particle (PP), particle-cluster
// (PC: targets of T, proxies of S), cluster-particle (CP) and
// cluster-cluster (CC); otherwise it splits the larger node, and two leaves
// that fail the test interact directly.  Every (target, source) pair is
// covered by exactly one interaction (check_coverage verifies it).
#pragma once
#include <cstdint>
#include <vector>

namespace bie {
namespace tree {

constexpr int kMaxP = 16;          // interpolation nodes per dimension
constexpr int kMaxProxies = 2048;  // proxies per cluster

struct Params {
  double theta = 0.5;   // acceptance: r_T + r_S < theta |c_T - c_S|
  int p = 8;            // nodes along a cluster's longest side (Laplace)
  double k = 0.0;       // |Re zk|: Helmholtz grids add nodes with k * side
  double kscale = 1.0;  // nodes added per radian of k * side / 2
  int leaf_t = 128;     // targets per target leaf (one thread block each)
  int leaf_s = 256;     // sources per source leaf
};

struct Node {
  int64_t b = 0, e = 0;        // point range in sorted order
  double lo[3] = {0, 0, 0};    // tight bounding box
  double hi[3] = {0, 0, 0};
  double c[3] = {0, 0, 0};     // box centre
  double r = 0;                // half diagonal
  int parent = -1, child0 = -1, nchild = 0, level = 0;
  int np[3] = {0, 0, 0};       // proxy grid; all 0 when the node has none
  bool capped = false;         // its grid would exceed kMaxP / kMaxProxies
  int64_t n() const { return e - b; }
  int nprox() const { return np[0] * np[1] * np[2]; }
};

struct Tree {
  std::vector<int64_t> perm;  // sorted position -> original index
  std::vector<Node> nodes;    // nodes[0] is the root; siblings are contiguous
};

// Builds the tree of n points (leaves hold at most `leaf` points unless the
// points coincide; siblings are contiguous, children follow their parents).
void build_tree(int64_t n, const double* x, const double* y, const double* z, int leaf, Tree& t);

// Chooses each node's proxy grid: along side d, np_d nodes such that the
// Chebyshev interpolation error for a source at the smallest accepted
// distance (r / theta) matches that of p nodes along the longest side,
// plus kscale * k * side_d / 2 for the oscillation of e^{ikr}; a node whose
// grid would hold as many points as the node itself gets none, and a node
// whose grid would exceed kMaxP points per side or kMaxProxies points gets
// none and is marked capped (the traversal then splits it rather than
// accept its pairs).
void set_proxies(Tree& t, const Params& prm);

enum Kind { kPPCheck = 0, kPP = 1, kPC = 2, kCP = 3, kCC = 4 };
struct Interaction {
  int t, s, kind;
};

// Dual traversal.  sep_min: accepted PP pairs whose boxes are closer than
// this keep the self-interaction test (kPPCheck).
void traverse(const Tree& T, const Tree& S, const Params& prm, double sep_min,
              std::vector<Interaction>& out);

// 0 when every (target leaf, source leaf) pair is covered exactly once.
int check_coverage(const Tree& T, const Tree& S, const std::vector<Interaction>& ia);

// Chebyshev points of the second kind on [-1, 1], cos(pi j / (p - 1))
// (the single point 0 when p = 1), and the Lagrange normalisations
// 1 / prod_{i != j} (x_j - x_i).
void cheb_nodes(int p, double* x, double* w);

}  // namespace tree
}  // namespace bie
