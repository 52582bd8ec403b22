// Deterministic graph bisection used for the hierarchical interface
// decomposition (HID) of AMSED / GMSLR.
//
// The reference calls METIS_PartGraphRecursive / METIS_PartGraphKway with two
// parts (include/utils/ExternalTools/MetisTools.h:173-180).  METIS is not part
// of the reference sources, so this file defines the partition instead, and
// the reference checker build links the same function behind a `metis.h`
// stand-in: both sides then consume identical partitions.
//
// Algorithm (level-structure bisection, George & Liu): find a
// pseudo-peripheral vertex by repeated breadth-first search from the
// minimum-degree vertex of the last level, then assign the first ceil(n/2)
// vertices of the breadth-first order from it to part 0 and the rest to
// part 1.  Every BFS visits neighbours in adjacency order, so the result only
// depends on the graph.
#include <cstdint>
#include <vector>

extern "C" {

// xadj[n+1], adjncy[xadj[n]] (0-based, no self loops required; self loops ignored).
// part[n] receives 0/1.  Returns the number of cut edges (each undirected edge counted once
// per direction, as METIS' edgecut counts adjacency entries / 2 would; here: adjacency
// entries crossing the cut).
int64_t prism_graph_bisect(int32_t n, const int32_t* xadj, const int32_t* adjncy, int32_t* part) {
    if (n <= 0) return 0;
    std::vector<int32_t> order(n), level(n, -1), deg(n, 0);
    for (int32_t v = 0; v < n; ++v)
        for (int32_t k = xadj[v]; k < xadj[v + 1]; ++k)
            if (adjncy[k] != v) deg[v]++;
    // BFS from `root` over the component; returns number of levels, fills order/level
    auto bfs = [&](int32_t root, int32_t& count) {
        for (int32_t i = 0; i < count; ++i) level[order[i]] = -1;
        count = 0;
        order[count++] = root;
        level[root] = 0;
        int32_t head = 0, nlev = 1;
        while (head < count) {
            const int32_t v = order[head++];
            for (int32_t k = xadj[v]; k < xadj[v + 1]; ++k) {
                const int32_t u = adjncy[k];
                if (level[u] < 0) {
                    level[u] = level[v] + 1;
                    if (level[u] + 1 > nlev) nlev = level[u] + 1;
                    order[count++] = u;
                }
            }
        }
        return nlev;
    };
    std::vector<int32_t> seen(n, 0);
    for (int32_t v = 0; v < n; ++v) part[v] = 1;
    // vertices are processed component by component in increasing index order;
    // the first half of the overall visiting order goes to part 0
    int32_t assigned0 = 0;
    const int32_t half = (n + 1) / 2;
    int32_t count = 0;
    for (int32_t start = 0; start < n; ++start) {
        if (seen[start]) continue;
        int32_t root = start;
        int32_t nlev = bfs(root, count);
        for (int guard = 0; guard < 64; ++guard) {
            // minimum-degree vertex of the last level
            int32_t best = -1;
            for (int32_t i = 0; i < count; ++i) {
                const int32_t u = order[i];
                if (level[u] == nlev - 1 && (best < 0 || deg[u] < deg[best])) best = u;
            }
            int32_t c2 = count;
            const int32_t nl2 = bfs(best, c2);
            count = c2;
            if (nl2 <= nlev) {
                root = best;
                break;
            }
            nlev = nl2;
            root = best;
        }
        nlev = bfs(root, count);
        for (int32_t i = 0; i < count; ++i) {
            const int32_t u = order[i];
            seen[u] = 1;
            if (assigned0 < half) {
                part[u] = 0;
                ++assigned0;
            }
        }
        for (int32_t i = 0; i < count; ++i) level[order[i]] = -1;
        count = 0;
    }
    int64_t cut = 0;
    for (int32_t v = 0; v < n; ++v)
        for (int32_t k = xadj[v]; k < xadj[v + 1]; ++k)
            if (part[adjncy[k]] != part[v]) ++cut;
    return cut / 2;
}

}  // extern "C"
