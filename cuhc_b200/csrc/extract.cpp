// HDBSCAN cluster extraction on the host: stability, cluster selection
// (excess of mass or leaves, optional epsilon merging, max cluster size),
// labels and membership probabilities of a condensed tree.
//
// Restates scikit-learn 1.9.0's sklearn/cluster/_hdbscan/_tree.pyx
// (_compute_stability, _get_clusters, epsilon_search, traverse_upwards,
// _do_labelling, get_probabilities, max_lambdas), the extraction the
// reference ports to NumPy (python/cuhc/_hdbscan.py:148-350), with the same
// float64 operations in the same order, so labels and probabilities are
// identical to sklearn's on the same tree:
//   stability(C) = sum over C's rows, in row order, of
//                  (lambda - birth(C)) * child size;
//   EOM, bottom-up over cluster ids: keep C unless its children's summed
//   stability exceeds its own (or C is larger than max_cluster_size); else
//   pass the sum up;
//   labels: each point takes its nearest selected ancestor (sklearn's
//   union-find over non-selected rows gives exactly that, since rows come
//   parent before child); probabilities: min(lambda, death) / death.
// The epsilon search does not depend on the order in which the selected
// clusters are visited: lambda never decreases down the tree, so the
// ancestor each leaf climbs to is either shared or disjoint.
#include <algorithm>
#include <cmath>
#include <map>
#include <set>
#include <vector>

#include "rnn.cuh"

namespace cuhc {
namespace {

using ll = long long;

struct CondensedTree {
  std::vector<ll> parent, child, size;
  std::vector<double> lambda;
  ll root = 0;
};

struct ClusterTree {
  // Rows with child size > 1 (cluster children), in condensed row order.
  std::vector<ll> parent, child, size;
  std::vector<double> lambda;
  std::map<ll, std::vector<ll>> children; // parent -> child clusters, row order
  std::map<ll, size_t> rowOfChild;        // cluster -> its row
};

ClusterTree clusterRows(const CondensedTree &t) {
  ClusterTree c;
  for (size_t i = 0; i < t.parent.size(); ++i) {
    if (t.size[i] <= 1)
      continue;
    c.rowOfChild[t.child[i]] = c.parent.size();
    c.parent.push_back(t.parent[i]);
    c.child.push_back(t.child[i]);
    c.size.push_back(t.size[i]);
    c.lambda.push_back(t.lambda[i]);
    c.children[t.parent[i]].push_back(t.child[i]);
  }
  return c;
}

void descendants(const ClusterTree &c, ll node, std::vector<ll> &out) {
  out.clear();
  out.push_back(node);
  for (size_t head = 0; head < out.size(); ++head) {
    auto it = c.children.find(out[head]);
    if (it != c.children.end())
      for (ll ch : it->second)
        out.push_back(ch);
  }
}

// The cluster a leaf with too small a split distance is replaced by.
ll climb(const ClusterTree &c, double epsilon, ll leaf, bool allowSingle) {
  const ll root = *std::min_element(c.parent.begin(), c.parent.end());
  while (true) {
    const ll parent = c.parent[c.rowOfChild.at(leaf)];
    if (parent == root)
      return allowSingle ? parent : leaf;
    const double parentEps = 1.0 / c.lambda[c.rowOfChild.at(parent)];
    if (parentEps > epsilon)
      return parent;
    leaf = parent;
  }
}

std::set<ll> epsilonSearch(const std::vector<ll> &leaves, const ClusterTree &c, double epsilon,
                           bool allowSingle) {
  std::set<ll> selected, processed;
  std::vector<ll> sub;
  for (ll leaf : leaves) {
    const double eps = 1.0 / c.lambda[c.rowOfChild.at(leaf)];
    if (eps < epsilon) {
      if (processed.count(leaf))
        continue;
      const ll top = climb(c, epsilon, leaf, allowSingle);
      selected.insert(top);
      descendants(c, top, sub);
      for (ll s : sub)
        if (s != top)
          processed.insert(s);
    } else {
      selected.insert(leaf);
    }
  }
  return selected;
}

void leavesBelow(const ClusterTree &c, ll node, std::vector<ll> &out) {
  auto it = c.children.find(node);
  if (it == c.children.end() || it->second.empty()) {
    out.push_back(node);
    return;
  }
  for (ll ch : it->second)
    leavesBelow(c, ch, out);
}

} // namespace

int hdbscanLabels(const double *tree, ll n, ll minClusterSize, int method, bool allowSingle,
                  double epsilon, ll maxClusterSize, ll *labels, double *probabilities) {
  if (n < 2) {
    for (ll i = 0; i < n; ++i) {
      labels[i] = -1;
      probabilities[i] = 0.0;
    }
    return 0;
  }
  // Condense.
  const ll capacity = n + 2 * (n / std::max(minClusterSize, 1LL)) + 2;
  CondensedTree t;
  t.parent.resize(capacity);
  t.child.resize(capacity);
  t.size.resize(capacity);
  t.lambda.resize(capacity);
  const ll rows = condenseTree(tree, n, minClusterSize, capacity, t.parent.data(),
                               t.child.data(), t.lambda.data(), t.size.data());
  if (rows < 0)
    return kErrorTooLarge;
  t.parent.resize(rows);
  t.child.resize(rows);
  t.size.resize(rows);
  t.lambda.resize(rows);
  t.root = *std::min_element(t.parent.begin(), t.parent.end());
  const ll root = t.root;
  const ll maxParent = *std::max_element(t.parent.begin(), t.parent.end());
  const ll largestChild = std::max(*std::max_element(t.child.begin(), t.child.end()), root);

  // Stability, accumulated in row order.
  std::vector<double> birth(largestChild + 1, NAN);
  for (ll i = 0; i < rows; ++i)
    birth[t.child[i]] = t.lambda[i];
  birth[root] = 0.0;
  std::vector<double> stability(maxParent - root + 1, 0.0);
  for (ll i = 0; i < rows; ++i)
    stability[t.parent[i] - root] += (t.lambda[i] - birth[t.parent[i]]) * (double)t.size[i];
  auto stab = [&](ll c) -> double & { return stability[c - root]; };

  // Clusters bottom-up: ids are a topological order (children > parents).
  std::vector<ll> nodes;
  for (ll c = maxParent; c >= root; --c)
    nodes.push_back(c);
  if (!allowSingle)
    nodes.pop_back(); // not the root
  const ClusterTree ct = clusterRows(t);
  ll samples = 0;
  for (ll i = 0; i < rows; ++i)
    if (t.size[i] == 1)
      samples = std::max(samples, t.child[i] + 1);
  const ll maxSize = maxClusterSize > 0 ? maxClusterSize : samples + 1;
  std::map<ll, ll> clusterSize;
  for (size_t i = 0; i < ct.child.size(); ++i)
    clusterSize[ct.child[i]] = ct.size[i];
  if (allowSingle && !nodes.empty()) {
    ll total = 0;
    for (size_t i = 0; i < ct.parent.size(); ++i)
      if (ct.parent[i] == nodes.back())
        total += ct.size[i];
    clusterSize[nodes.back()] = total;
  }
  std::map<ll, bool> isCluster;
  for (ll c : nodes)
    isCluster[c] = true;
  std::vector<ll> sub;
  if (method == 0) { // excess of mass
    for (ll node : nodes) {
      double subtree = 0.0;
      auto it = ct.children.find(node);
      bool first = true;
      if (it != ct.children.end())
        for (ll ch : it->second) {
          subtree = first ? stab(ch) : subtree + stab(ch);
          first = false;
        }
      if (subtree > stab(node) || clusterSize[node] > maxSize) {
        isCluster[node] = false;
        stab(node) = subtree;
      } else {
        descendants(ct, node, sub);
        for (ll s : sub)
          if (s != node)
            isCluster[s] = false;
      }
    }
    if (epsilon != 0.0 && !ct.parent.empty()) {
      std::vector<ll> eom;
      for (ll c : nodes)
        if (isCluster[c])
          eom.push_back(c);
      const ll ctRoot = *std::min_element(ct.parent.begin(), ct.parent.end());
      std::set<ll> selected;
      if (eom.size() == 1 && eom[0] == ctRoot) {
        if (allowSingle)
          selected.insert(eom[0]);
      } else {
        selected = epsilonSearch(eom, ct, epsilon, allowSingle);
      }
      for (auto &kv : isCluster)
        kv.second = selected.count(kv.first) > 0;
    }
  } else { // leaves
    std::vector<ll> leaves;
    if (!ct.parent.empty())
      leavesBelow(ct, *std::min_element(ct.parent.begin(), ct.parent.end()), leaves);
    std::set<ll> selected;
    if (epsilon != 0.0)
      selected = epsilonSearch(leaves, ct, epsilon, allowSingle);
    else
      selected.insert(leaves.begin(), leaves.end());
    for (auto &kv : isCluster)
      kv.second = selected.count(kv.first) > 0;
  }
  std::vector<ll> clusters;
  for (auto &kv : isCluster)
    if (kv.second)
      clusters.push_back(kv.first);
  std::sort(clusters.begin(), clusters.end());
  std::map<ll, ll> labelOf;
  for (size_t i = 0; i < clusters.size(); ++i)
    labelOf[clusters[i]] = (ll)i;

  // Labels: nearest selected ancestor, propagated top-down over the rows.
  std::vector<ll> owner(maxParent + 1, -1);
  owner[root] = root;
  for (ll i = 0; i < rows; ++i) {
    const ll c = t.child[i];
    if (t.size[i] > 1)
      owner[c] = labelOf.count(c) ? c : owner[t.parent[i]];
  }
  for (ll p = 0; p < root; ++p)
    labels[p] = -1;
  const bool singleRoot = clusters.size() == 1 && allowSingle;
  double rootThreshold = 0.0;
  if (singleRoot) {
    if (epsilon != 0.0) {
      rootThreshold = 1.0 / epsilon;
    } else {
      rootThreshold = -INFINITY;
      for (ll i = 0; i < rows; ++i)
        if (t.parent[i] == root)
          rootThreshold = std::max(rootThreshold, t.lambda[i]);
    }
  }
  for (ll i = 0; i < rows; ++i) {
    const ll pnt = t.child[i];
    if (pnt >= root)
      continue;
    const ll own = owner[t.parent[i]];
    if (own != root) {
      labels[pnt] = labelOf[own];
    } else if (singleRoot && labelOf.count(root) && t.lambda[i] >= rootThreshold) {
      labels[pnt] = labelOf[root];
    }
  }

  // Probabilities: deaths are the run maxima of consecutive equal parents.
  std::vector<double> death(maxParent + 1, 0.0);
  ll current = t.parent[0];
  double runMax = t.lambda[0];
  for (ll i = 1; i < rows; ++i) {
    if (t.parent[i] == current) {
      runMax = std::max(runMax, t.lambda[i]);
    } else {
      death[current] = runMax;
      current = t.parent[i];
      runMax = t.lambda[i];
    }
  }
  death[current] = runMax;
  for (ll p = 0; p < root; ++p)
    probabilities[p] = 0.0;
  for (ll i = 0; i < rows; ++i) {
    const ll pnt = t.child[i];
    if (pnt >= root || labels[pnt] == -1)
      continue;
    const double maxLambda = death[clusters[labels[pnt]]];
    if (maxLambda == 0.0 || std::isinf(t.lambda[i]))
      probabilities[pnt] = 1.0;
    else
      probabilities[pnt] = std::min(t.lambda[i], maxLambda) / maxLambda;
  }
  return 0;
}

} // namespace cuhc

extern "C" {

// Labels (-1 = noise) and membership probabilities of HDBSCAN's clustering
// of a (n-1) x 4 single-linkage tree. method: 0 excess of mass, 1 leaf;
// maxClusterSize <= 0 means no limit. No counterpart in the reference's C
// ABI (its extraction is NumPy, python/cuhc/_hdbscan.py:148-350).
int cuhc_hdbscan_labels(const double *tree, long long n, long long minClusterSize, int method,
                        int allowSingleCluster, double epsilon, long long maxClusterSize,
                        long long *labels, double *probabilities) {
  if (n <= 0 || minClusterSize < 1)
    return cuhc::kErrorInvalidShape;
  if (method < 0 || method > 1)
    return cuhc::kErrorInvalidAlgorithm;
  return cuhc::hdbscanLabels(tree, n, minClusterSize, method, allowSingleCluster != 0, epsilon,
                             maxClusterSize, labels, probabilities);
}

} // extern "C"
