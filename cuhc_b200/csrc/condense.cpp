// HDBSCAN's condensed tree (host). Walks the scipy-format single-linkage tree
// breadth-first from the root with sklearn 1.9's rules, emitting rows in the
// same order as sklearn's _condense_tree and the reference's condenseTree
// (hdbscan.cuh:398-483):
//   both children >= minClusterSize   two new clusters split off;
//   one child smaller                 the larger child continues the parent
//                                     cluster; the smaller child's points
//                                     fall out of it, breadth-first;
//   both smaller                      all points fall out, left then right.
#include <cmath>
#include <vector>

#include "rnn.cuh"

namespace cuhc {

namespace {

struct TreeView {
  const double *z;
  long long n;
  long long left(long long node) const { return (long long)z[(node - n) * 4 + 0]; }
  long long right(long long node) const { return (long long)z[(node - n) * 4 + 1]; }
  double height(long long node) const { return z[(node - n) * 4 + 2]; }
  long long count(long long node) const {
    return node >= n ? (long long)z[(node - n) * 4 + 3] : 1;
  }
};

// Nodes below `from`, breadth-first, children left then right.
void breadthFirst(const TreeView &t, long long from, std::vector<long long> &out) {
  out.clear();
  out.push_back(from);
  for (size_t head = 0; head < out.size(); ++head) {
    const long long node = out[head];
    if (node >= t.n) {
      out.push_back(t.left(node));
      out.push_back(t.right(node));
    }
  }
}

} // namespace

long long condenseTree(const double *tree, long long n, long long minClusterSize,
                       long long capacity, long long *parent, long long *child, double *lambda,
                       long long *size) {
  if (n < 2)
    return 0;
  const TreeView t{tree, n};
  const long long root = 2 * (n - 1);
  std::vector<long long> nodes, subtree;
  breadthFirst(t, root, nodes);
  std::vector<long long> label(root + 1, 0);
  std::vector<char> done(root + 1, 0);
  label[root] = n;
  long long nextLabel = n + 1, rows = 0;
  auto emit = [&](long long p, long long c, double l, long long s) {
    if (rows < capacity) {
      parent[rows] = p;
      child[rows] = c;
      lambda[rows] = l;
      size[rows] = s;
    }
    ++rows;
  };
  auto fallOut = [&](long long parentLabel, long long from, double l) {
    breadthFirst(t, from, subtree);
    for (long long node : subtree) {
      if (node < n)
        emit(parentLabel, node, l, 1);
      done[node] = 1;
    }
  };
  for (long long node : nodes) {
    if (node < n || done[node])
      continue;
    const long long a = t.left(node), b = t.right(node);
    const double h = t.height(node);
    const double l = h > 0.0 ? 1.0 / h : INFINITY;
    const long long ca = t.count(a), cb = t.count(b);
    const bool bigA = ca >= minClusterSize, bigB = cb >= minClusterSize;
    if (bigA && bigB) {
      label[a] = nextLabel++;
      emit(label[node], label[a], l, ca);
      label[b] = nextLabel++;
      emit(label[node], label[b], l, cb);
      continue;
    }
    if (bigA)
      label[a] = label[node];
    else
      fallOut(label[node], a, l);
    if (bigB)
      label[b] = label[node];
    else
      fallOut(label[node], b, l);
  }
  return rows <= capacity ? rows : -rows;
}

} // namespace cuhc
