// Community ordering of a graph's vertices for locality (cola_community_order):
// the reordering step CoLa runs before partitioning (rabbit_order_write.py
// calls the Rabbit Order module, rabbit_module/src/reorder.cpp:260-288), written
// here from the published method (J. Arai et al., "Rabbit Order: Just-in-Time
// Parallel Reordering for Fast Graph Analysis", IPDPS 2016), sequentially:
//
//  1. Community detection by incremental aggregation.  Every vertex starts as
//     its own community.  Vertices are visited in increasing order of degree;
//     a visited vertex u gathers the edges of its community (its own and those
//     of the vertices merged into it earlier, each resolved to the community
//     it now belongs to) and merges into the neighbouring community v with the
//     largest modularity gain, dQ(u, v) = 2 (w_uv / 2m - d_u d_v / (2m)^2),
//     when that gain is positive; otherwise u stays a top-level community.
//     Each merge makes u a child of v in a dendrogram.
//  2. Ordering.  The top-level communities are taken in increasing order of
//     their vertex ids, and each dendrogram is walked depth first (a vertex,
//     then its children in merge order), numbering vertices as they are
//     reached, so that every community's vertices get consecutive ids and
//     communities merged early sit next to each other.
//
// The graph is taken as undirected: each COO entry (r, c), r != c, is an edge
// of weight 1 between r and c (both directions of a symmetric list count
// twice, which scales every weight alike); duplicates add up; self-loops are
// ignored.  Deterministic.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "common.h"
#include "prep.h"

namespace cola {

cola_status community_order(int32_t n, int64_t nnz, const int32_t *row, const int32_t *col, int32_t *mapping,
                            int64_t *communities)
{
    COLA_REQUIRE(n >= 0 && nnz >= 0 && (nnz == 0 || (row && col)) && (n == 0 || mapping), COLA_ERROR_INVALID_ARGUMENT,
                 "cola_community_order: bad arguments");
    for (int64_t i = 0; i < nnz; i++)
        COLA_REQUIRE(row[i] >= 0 && row[i] < n && col[i] >= 0 && col[i] < n, COLA_ERROR_INVALID_ARGUMENT,
                     "cola_community_order: entry %lld (%d, %d) outside %d vertices", (long long)i, row[i], col[i],
                     n);
    // undirected adjacency (both directions of every non-loop entry), CSR
    std::vector<int64_t> ptr((size_t)n + 1, 0);
    for (int64_t i = 0; i < nnz; i++)
        if (row[i] != col[i]) {
            ptr[(size_t)row[i] + 1]++;
            ptr[(size_t)col[i] + 1]++;
        }
    for (int32_t v = 0; v < n; v++)
        ptr[(size_t)v + 1] += ptr[(size_t)v];
    std::vector<int32_t> adj((size_t)ptr[(size_t)n]);
    {
        std::vector<int64_t> at(ptr.begin(), ptr.end() - 1);
        for (int64_t i = 0; i < nnz; i++)
            if (row[i] != col[i]) {
                adj[(size_t)at[(size_t)row[i]]++] = col[i];
                adj[(size_t)at[(size_t)col[i]]++] = row[i];
            }
    }
    std::vector<double> tot((size_t)n);  // community degree (sum of edge weights)
    for (int32_t v = 0; v < n; v++)
        tot[(size_t)v] = (double)(ptr[(size_t)v + 1] - ptr[(size_t)v]);
    const double m2 = (double)ptr[(size_t)n];  // 2m

    // union-find parent (the community a merged vertex joined), dendrogram
    // children (first child / next sibling, in merge order), and the
    // aggregated edge list a visited vertex leaves for its community
    std::vector<int32_t> parent((size_t)n), first((size_t)n, -1), last((size_t)n, -1), next((size_t)n, -1);
    std::iota(parent.begin(), parent.end(), 0);
    std::vector<std::vector<std::pair<int32_t, double>>> agg((size_t)n);
    auto find = [&](int32_t x) {
        int32_t r = x;
        while (parent[(size_t)r] != r)
            r = parent[(size_t)r];
        while (parent[(size_t)x] != r) {  // path compression
            const int32_t p = parent[(size_t)x];
            parent[(size_t)x] = r;
            x = p;
        }
        return r;
    };

    std::vector<int32_t> order((size_t)n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return ptr[(size_t)a + 1] - ptr[(size_t)a] < ptr[(size_t)b + 1] - ptr[(size_t)b];
    });
    std::vector<double> wacc((size_t)n, 0.0);
    std::vector<int32_t> touched;
    for (int32_t u : order) {
        if (parent[(size_t)u] != u)
            continue;  // already merged into another community
        touched.clear();
        auto add = [&](int32_t x, double w) {
            const int32_t r = find(x);
            if (r == u)
                return;
            if (wacc[(size_t)r] == 0.0)
                touched.push_back(r);
            wacc[(size_t)r] += w;
        };
        for (int64_t q = ptr[(size_t)u]; q < ptr[(size_t)u + 1]; q++)
            add(adj[(size_t)q], 1.0);
        for (int32_t c = first[(size_t)u]; c >= 0; c = next[(size_t)c]) {
            for (const auto &e : agg[(size_t)c])
                add(e.first, e.second);
            std::vector<std::pair<int32_t, double>>().swap(agg[(size_t)c]);
        }
        std::sort(touched.begin(), touched.end());  // ties go to the smallest community id
        int32_t best = -1;
        double gain = 0.0;
        for (int32_t r : touched) {
            const double g = wacc[(size_t)r] / m2 - tot[(size_t)u] * tot[(size_t)r] / (m2 * m2);
            if (g > gain) {
                gain = g;
                best = r;
            }
        }
        std::vector<std::pair<int32_t, double>> mine;
        mine.reserve(touched.size());
        for (int32_t r : touched) {
            mine.emplace_back(r, wacc[(size_t)r]);
            wacc[(size_t)r] = 0.0;
        }
        if (best >= 0) {
            parent[(size_t)u] = best;
            tot[(size_t)best] += tot[(size_t)u];
            if (last[(size_t)best] < 0)
                first[(size_t)best] = u;
            else
                next[(size_t)last[(size_t)best]] = u;
            last[(size_t)best] = u;
            agg[(size_t)u] = std::move(mine);  // read when `best` is visited
        }
    }

    // number the vertices: top-level communities by id, each dendrogram depth first
    int32_t id = 0;
    int64_t ncomm = 0;
    std::vector<int32_t> stack;
    for (int32_t v = 0; v < n; v++) {
        if (parent[(size_t)v] != v)
            continue;
        ncomm++;
        stack.push_back(v);
        while (!stack.empty()) {
            const int32_t x = stack.back();
            stack.pop_back();
            mapping[(size_t)x] = id++;
            // children pushed last-first, so they are reached in merge order
            std::vector<int32_t> kids;
            for (int32_t c = first[(size_t)x]; c >= 0; c = next[(size_t)c])
                kids.push_back(c);
            for (size_t k = kids.size(); k-- > 0;)
                stack.push_back(kids[k]);
        }
    }
    if (communities)
        *communities = ncomm;
    return COLA_SUCCESS;
}

}  // namespace cola

extern "C" cola_status cola_community_order(int32_t num_nodes, int64_t nnz, const int32_t *row, const int32_t *col,
                                            int32_t *mapping, int64_t *communities)
{
    cola::clear_error();
    return cola::community_order(num_nodes, nnz, row, col, mapping, communities);
}
