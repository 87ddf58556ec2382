// Balanced compact node partition (see hsc_partition.h).
#include "hsc_partition.h"

#include <algorithm>
#include <cstdint>
#include <functional>
#include <queue>
#include <utility>

namespace hsc {

namespace {

struct Graph {
    int n;
    const std::vector<int>& ptr;
    const std::vector<int>& adj;
};

// breadth-first distances from `src` (several sources allowed), restricted to
// nodes with mask[v] == tag; -1 elsewhere.  Visits in index order per layer.
void bfs(const Graph& g, const std::vector<int>& src, const std::vector<int>& mask, int tag, std::vector<int>& dist,
         std::vector<int>& touched) {
    for (int v : touched) dist[v] = -1;
    touched.clear();
    std::vector<int> cur, nxt;
    for (int s : src)
        if (dist[s] < 0 && mask[s] == tag) { dist[s] = 0; cur.push_back(s); touched.push_back(s); }
    int d = 0;
    while (!cur.empty()) {
        ++d;
        nxt.clear();
        for (int u : cur)
            for (int e = g.ptr[u]; e < g.ptr[u + 1]; ++e) {
                const int v = g.adj[e];
                if (dist[v] < 0 && mask[v] == tag) { dist[v] = d; nxt.push_back(v); touched.push_back(v); }
            }
        std::sort(nxt.begin(), nxt.end());
        cur.swap(nxt);
    }
}

// grow all parts from their seeds: the lightest part (ties: lower id) takes the
// next free node of its own breadth-first front (a FIFO, so its nearest free
// neighbour; ties in insertion order); nodes no part reached (none in a connected
// component with a seed) are left -1
void grow(const Graph& g, const std::vector<double>& w, const std::vector<int>& seeds, std::vector<int>& part) {
    const int P = (int)seeds.size();
    std::fill(part.begin(), part.end(), -1);
    std::vector<std::vector<int>> front(P);
    std::vector<size_t> head(P, 0);
    using PW = std::pair<double, int>;
    std::priority_queue<PW, std::vector<PW>, std::greater<PW>> parts;
    std::vector<double> load(P, 0.0);
    for (int p = 0; p < P; ++p) {
        front[p].push_back(seeds[p]);
        parts.push({0.0, p});
    }
    while (!parts.empty()) {
        const int p = parts.top().second;
        parts.pop();
        auto& f = front[p];
        size_t& h = head[p];
        while (h < f.size() && part[f[h]] >= 0) ++h;
        if (h == f.size()) continue;  // enclosed: the part stops growing
        const int u = f[h++];
        part[u] = p;
        load[p] += w[u];
        for (int e = g.ptr[u]; e < g.ptr[u + 1]; ++e)
            if (part[g.adj[e]] < 0) f.push_back(g.adj[e]);
        parts.push({load[p], p});
    }
}

}  // namespace

std::vector<int> partition_nodes(int n, const std::vector<int>& adj_ptr, const std::vector<int>& adj,
                                 const std::vector<double>& weight, int nparts) {
    std::vector<int> part(n, 0);
    if (n <= 0 || nparts <= 1) return part;
    nparts = std::min(nparts, n);
    const Graph g{n, adj_ptr, adj};
    // connected components
    std::vector<int> comp(n, -1);
    int ncomp = 0;
    {
        std::vector<int> stack;
        for (int s = 0; s < n; ++s) {
            if (comp[s] >= 0) continue;
            comp[s] = ncomp;
            stack.push_back(s);
            while (!stack.empty()) {
                const int u = stack.back();
                stack.pop_back();
                for (int e = adj_ptr[u]; e < adj_ptr[u + 1]; ++e)
                    if (comp[adj[e]] < 0) { comp[adj[e]] = ncomp; stack.push_back(adj[e]); }
            }
            ++ncomp;
        }
    }
    // parts per component in proportion to weight (largest remainders), at least one each;
    // with more components than parts, components are packed whole onto the lightest part
    std::vector<double> cw(ncomp, 0.0);
    std::vector<int> csize(ncomp, 0);
    double tot = 0.0;
    for (int i = 0; i < n; ++i) { cw[comp[i]] += weight[i]; csize[comp[i]]++; tot += weight[i]; }
    if (ncomp >= nparts) {
        std::vector<int> order(ncomp);
        for (int c = 0; c < ncomp; ++c) order[c] = c;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cw[a] > cw[b]; });
        std::vector<double> load(nparts, 0.0);
        std::vector<int> cpart(ncomp, 0);
        for (int c : order) {
            const int p = (int)(std::min_element(load.begin(), load.end()) - load.begin());
            cpart[c] = p;
            load[p] += cw[c];
        }
        for (int i = 0; i < n; ++i) part[i] = cpart[comp[i]];
        return part;
    }
    std::vector<int> alloc(ncomp, 1);
    {
        int used = ncomp;
        std::vector<double> rem(ncomp);
        for (int c = 0; c < ncomp; ++c) {
            const double share = cw[c] / tot * nparts;
            const int extra = std::max(0, std::min(csize[c], (int)share) - 1);
            alloc[c] += extra;
            used += extra;
            rem[c] = share - alloc[c];
        }
        while (used < nparts) {
            int best = -1;
            for (int c = 0; c < ncomp; ++c)
                if (alloc[c] < csize[c] && (best < 0 || rem[c] > rem[best])) best = c;
            if (best < 0) break;
            alloc[best]++;
            rem[best] -= 1.0;
            ++used;
        }
    }
    // seeds: farthest-point sampling by breadth-first distance inside each component.  near[v] is
    // the distance to the nearest seed so far; a new seed only re-labels the nodes it is closer to
    // (a breadth-first pass that stops where it does not improve), then the farthest node is next.
    std::vector<int> seeds;
    std::vector<int> dist(n, -1), touched;
    std::vector<std::vector<int>> members(ncomp);
    for (int i = 0; i < n; ++i) members[comp[i]].push_back(i);
    std::vector<int> near(n, 1 << 30), queue;
    for (int c = 0; c < ncomp; ++c) {
        const std::vector<int>& mem = members[c];
        bfs(g, {mem[0]}, comp, c, dist, touched);
        int s = mem[0];
        for (int v : touched)
            if (dist[v] > dist[s] || (dist[v] == dist[s] && v < s)) s = v;
        for (int k = 0; k < alloc[c]; ++k) {
            seeds.push_back(s);
            near[s] = 0;
            queue.assign(1, s);
            for (size_t h = 0; h < queue.size(); ++h) {
                const int u = queue[h];
                for (int e = adj_ptr[u]; e < adj_ptr[u + 1]; ++e) {
                    const int v = adj[e];
                    if (near[u] + 1 < near[v]) { near[v] = near[u] + 1; queue.push_back(v); }
                }
            }
            int far = mem[0];
            for (int v : mem)
                if (near[v] > near[far]) far = v;   // members ascend: ties keep the lower index
            s = far;
        }
    }
    grow(g, weight, seeds, part);
    for (int i = 0; i < n; ++i)
        if (part[i] < 0) part[i] = 0;  // unreachable: every component has a seed
    // balance: growth stops a part when its neighbours enclose it, so parts where the seeds sat
    // sparse end up heavy.  Sweeps let weight flow downhill: a boundary node of a part above its
    // component's mean (+2 %) moves to the lightest neighbouring part that is lighter by more than
    // twice the node's weight, when the node has at least half as many neighbours there as it
    // keeps (no long thin fingers); repeated until no node moves.  Moves follow edges, so parts stay
    // inside their component.
    {
        const int P = (int)seeds.size();
        std::vector<double> load(P, 0.0);
        for (int i = 0; i < n; ++i) load[part[i]] += weight[i];
        std::vector<int> pcomp(P, 0);
        for (int i = 0; i < n; ++i) pcomp[part[i]] = comp[i];
        std::vector<int> nbp;
        for (int sweep = 0; sweep < 64; ++sweep) {
            int moved = 0;
            for (int u = 0; u < n; ++u) {
                const int p = part[u];
                if (load[p] <= 1.02 * cw[pcomp[p]] / alloc[pcomp[p]]) continue;
                nbp.clear();
                int own = 0;
                for (int e = adj_ptr[u]; e < adj_ptr[u + 1]; ++e) {
                    const int q = part[adj[e]];
                    if (q == p) ++own;
                    else nbp.push_back(q);
                }
                if (nbp.empty()) continue;
                std::sort(nbp.begin(), nbp.end());
                int best = -1;
                for (size_t i = 0; i < nbp.size();) {
                    size_t j = i;
                    while (j < nbp.size() && nbp[j] == nbp[i]) ++j;
                    const int q = nbp[i], c = (int)(j - i);
                    if (2 * c >= own && load[q] + 2 * weight[u] < load[p] && (best < 0 || load[q] < load[best]))
                        best = q;
                    i = j;
                }
                if (best < 0) continue;
                part[u] = best;
                load[p] -= weight[u];
                load[best] += weight[u];
                ++moved;
            }
            if (!moved) break;
        }
    }
    return part;
}

}  // namespace hsc
