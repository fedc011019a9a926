#include "mas_ordering.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <omp.h>

namespace pmas
{
    std::vector<uint8_t> isolated_blocks(int n, const int *outer, const int *inner, int bd)
    {
        const int V = (n + bd - 1) / bd;
        std::vector<uint8_t> iso(V, 1);
        // A block column j/bd with an entry in another block row couples both blocks.
#pragma omp parallel for schedule(dynamic, 1024)
        for (int j = 0; j < n; ++j)
        {
            const int bj = j / bd;
            for (int k = outer[j]; k < outer[j + 1]; ++k)
            {
                const int bi = inner[k] / bd;
                if (bi != bj)
                {
                    iso[bi] = 0; // benign race: every writer stores 0
                    iso[bj] = 0;
                }
            }
        }
        return iso;
    }

    namespace
    {
        inline uint64_t spread3(uint64_t v)
        {
            v &= 0x1FFFFFull;
            v = (v | (v << 32)) & 0x1F00000000FFFFull;
            v = (v | (v << 16)) & 0x1F0000FF0000FFull;
            v = (v | (v << 8)) & 0x100F00F00F00F00Full;
            v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
            v = (v | (v << 2)) & 0x1249249249249249ull;
            return v;
        }

        // Nodes in `order` (coupled ones first) -> padded ids: coupled chunked by 32 from bank 0,
        // isolated ones from the next bank boundary.
        std::vector<int> assign_padded(const std::vector<int> &order, int nreal, int *banks)
        {
            const int V = (int)order.size();
            std::vector<int> padded(V);
            for (int t = 0; t < nreal; ++t)
                padded[order[t]] = t;
            const int base = (nreal + 31) / 32 * 32;
            for (int t = nreal; t < V; ++t)
                padded[order[t]] = base + (t - nreal);
            const int niso = V - nreal;
            *banks = (nreal + 31) / 32 + (niso + 31) / 32;
            return padded;
        }
    } // namespace

    std::vector<int> morton_padded(const double *xyz, int V, const std::vector<uint8_t> &isolated, int *banks)
    {
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        if (V > 0)
            for (int d = 0; d < 3; ++d)
                lo[d] = hi[d] = xyz[d];
        for (int v = 0; v < V; ++v)
            for (int d = 0; d < 3; ++d)
            {
                lo[d] = std::min(lo[d], xyz[3 * (size_t)v + d]);
                hi[d] = std::max(hi[d], xyz[3 * (size_t)v + d]);
            }
        double ext[3];
        int ndims = 0;
        double vol = 1.0, emax = 0.0;
        for (int d = 0; d < 3; ++d)
        {
            ext[d] = hi[d] - lo[d];
            emax = std::max(emax, ext[d]);
            if (ext[d] > 0.0)
            {
                vol = vol * ext[d];
                ++ndims;
            }
        }
        double scale = 0.0;
        if (ndims > 0)
        {
            const double h = std::pow(vol / V, 1.0 / ndims);
            scale = std::min(1.0 / h, 2097151.0 / emax);
        }
        std::vector<uint64_t> code(V);
#pragma omp parallel for schedule(static)
        for (int v = 0; v < V; ++v)
        {
            uint64_t q[3];
            for (int d = 0; d < 3; ++d)
            {
                double f = (ndims > 0) ? std::floor((xyz[3 * (size_t)v + d] - lo[d]) * scale + 0.5) : 0.0;
                if (f < 0.0)
                    f = 0.0;
                if (f > 2097151.0)
                    f = 2097151.0;
                q[d] = (uint64_t)f;
            }
            code[v] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
        }
        std::vector<int> order(V);
        std::iota(order.begin(), order.end(), 0);
        std::sort(order.begin(), order.end(), [&](int a, int b) {
            if (isolated[a] != isolated[b])
                return isolated[a] < isolated[b];
            if (code[a] != code[b])
                return code[a] < code[b];
            return a < b;
        });
        int nreal = 0;
        for (int v = 0; v < V; ++v)
            nreal += isolated[v] ? 0 : 1;
        return assign_padded(order, nreal, banks);
    }

    namespace
    {
        struct Graph
        {
            std::vector<long long> ptr;
            std::vector<int> adj;
        };

        Graph block_graph(int n, const int *outer, const int *inner, int bd)
        {
            const int V = (n + bd - 1) / bd;
            std::vector<std::vector<int>> nb(V);
#pragma omp parallel for schedule(dynamic, 256)
            for (int bj = 0; bj < V; ++bj)
            {
                auto &lst = nb[bj];
                for (int j = bj * bd; j < std::min(n, (bj + 1) * bd); ++j)
                    for (int k = outer[j]; k < outer[j + 1]; ++k)
                    {
                        const int bi = inner[k] / bd;
                        if (bi != bj)
                            lst.push_back(bi);
                    }
                std::sort(lst.begin(), lst.end());
                lst.erase(std::unique(lst.begin(), lst.end()), lst.end());
            }
            Graph g;
            g.ptr.assign(V + 1, 0);
            for (int v = 0; v < V; ++v)
                g.ptr[v + 1] = g.ptr[v] + (long long)nb[v].size();
            g.adj.resize(g.ptr[V]);
#pragma omp parallel for schedule(static)
            for (int v = 0; v < V; ++v)
                std::copy(nb[v].begin(), nb[v].end(), g.adj.begin() + g.ptr[v]);
            return g;
        }

        // BFS distances inside the subset marked tag[v] == t, restarting at unvisited nodes so
        // every node of the subset gets a distance. Returns the last node reached.
        int bfs(const Graph &g, const std::vector<int> &nodes, int start, const std::vector<int> &tag, int t,
                std::vector<int> &dist, std::vector<int> &queue)
        {
            for (int v : nodes)
                dist[v] = -1;
            int last = start, base = 0;
            size_t next_seed = 0;
            queue.clear();
            int seed = start;
            for (;;)
            {
                dist[seed] = base;
                queue.push_back(seed);
                size_t head = queue.size() - 1;
                int maxd = base;
                while (head < queue.size())
                {
                    const int v = queue[head++];
                    last = v;
                    maxd = std::max(maxd, dist[v]);
                    for (long long k = g.ptr[v]; k < g.ptr[v + 1]; ++k)
                    {
                        const int w = g.adj[k];
                        if (tag[w] == t && dist[w] < 0)
                        {
                            dist[w] = dist[v] + 1;
                            queue.push_back(w);
                        }
                    }
                }
                if (queue.size() == nodes.size())
                    break;
                while (next_seed < nodes.size() && dist[nodes[next_seed]] >= 0)
                    ++next_seed;
                if (next_seed >= nodes.size())
                    break;
                seed = nodes[next_seed];
                base = maxd + 1;
            }
            return last;
        }

        void bisect(const Graph &g, std::vector<int> nodes, int t, std::vector<int> &tag, std::vector<int> &dist,
                    std::vector<int> &out, int &next_tag)
        {
            if (nodes.size() <= 32)
            {
                std::sort(nodes.begin(), nodes.end());
                out.insert(out.end(), nodes.begin(), nodes.end());
                return;
            }
            std::vector<int> queue;
            queue.reserve(nodes.size());
            std::sort(nodes.begin(), nodes.end());
            const int far = bfs(g, nodes, nodes[0], tag, t, dist, queue);
            bfs(g, nodes, far, tag, t, dist, queue);
            std::vector<std::pair<int, int>> key(nodes.size());
            for (size_t i = 0; i < nodes.size(); ++i)
                key[i] = {dist[nodes[i]], nodes[i]};
            std::sort(key.begin(), key.end());
            const size_t half = (nodes.size() + 1) / 2;
            const size_t k = std::min(nodes.size() - 1, (half + 31) / 32 * 32);
            std::vector<int> left(k), right(nodes.size() - k);
            for (size_t i = 0; i < k; ++i)
                left[i] = key[i].second;
            for (size_t i = k; i < nodes.size(); ++i)
                right[i - k] = key[i].second;
            const int tl = next_tag++, tr = next_tag++;
            for (int v : left)
                tag[v] = tl;
            for (int v : right)
                tag[v] = tr;
            bisect(g, std::move(left), tl, tag, dist, out, next_tag);
            bisect(g, std::move(right), tr, tag, dist, out, next_tag);
        }
    } // namespace

    std::vector<int> graph_padded(int n, const int *outer, const int *inner, int bd,
                                  const std::vector<uint8_t> &isolated, int *banks)
    {
        const int V = (n + bd - 1) / bd;
        Graph g = block_graph(n, outer, inner, bd);
        std::vector<int> coupled;
        for (int v = 0; v < V; ++v)
            if (!isolated[v])
                coupled.push_back(v);
        std::vector<int> tag(V, -1), dist(V, -1), order;
        order.reserve(V);
        for (int v : coupled)
            tag[v] = 0;
        int next_tag = 1;
        const int nreal = (int)coupled.size();
        if (nreal > 0)
            bisect(g, coupled, 0, tag, dist, order, next_tag);
        // Every left part has a multiple of 32 nodes, so all leaves but the last hold exactly 32
        // nodes and chunking the emitted sequence by 32 gives back the leaves.
        for (int v = 0; v < V; ++v)
            if (isolated[v])
                order.push_back(v);
        return assign_padded(order, nreal, banks);
    }

    std::vector<int> natural_padded(int V, int *banks)
    {
        std::vector<int> padded(V);
        std::iota(padded.begin(), padded.end(), 0);
        *banks = (V + 31) / 32;
        return padded;
    }

    uint64_t pattern_hash(int n, const int *outer, const int *inner, long long nnz, bool *valid, int threads)
    {
        // FNV-1a over 32-bit words, split into chunks (threads) and, inside a chunk, into eight
        // interleaved lanes (independent multiply chains: the loop runs at memory speed instead of
        // the multiplier's latency). Column pointers are hashed and checked in the same chunks.
        constexpr uint64_t OFFSET = 1469598103934665603ull, PRIME = 1099511628211ull;
        constexpr int chunks = 256, LANES = 8;
        std::vector<uint64_t> part(chunks, 0), opart(chunks, 0);
        std::vector<uint8_t> bad(chunks, 0);
        if (threads <= 0)
            threads = omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(threads)
        for (int c = 0; c < chunks; ++c)
        {
            const long long lo = nnz * c / chunks, hi = nnz * (c + 1) / chunks;
            uint64_t h[LANES];
            for (int l = 0; l < LANES; ++l)
                h[l] = OFFSET ^ (uint64_t)(c * LANES + l);
            uint32_t out_of_range = 0; // negative rows wrap to large unsigned values
            long long k = lo;
            for (; k + LANES <= hi; k += LANES)
                for (int l = 0; l < LANES; ++l)
                {
                    const uint32_t i = (uint32_t)inner[k + l];
                    out_of_range |= (uint32_t)(i >= (uint32_t)n);
                    h[l] = (h[l] ^ (uint64_t)i) * PRIME;
                }
            for (; k < hi; ++k)
            {
                const uint32_t i = (uint32_t)inner[k];
                out_of_range |= (uint32_t)(i >= (uint32_t)n);
                h[0] = (h[0] ^ (uint64_t)i) * PRIME;
            }
            uint64_t g = OFFSET;
            for (int l = 0; l < LANES; ++l)
                g = (g ^ h[l]) * PRIME;
            part[c] = g;
            // Column pointers j in [olo, ohi): hashed, and non-decreasing.
            const long long olo = (long long)(n + 1) * c / chunks, ohi = (long long)(n + 1) * (c + 1) / chunks;
            uint64_t ho = OFFSET ^ (uint64_t)c;
            bool decreasing = false;
            for (long long j = olo; j < ohi; ++j)
            {
                ho = (ho ^ (uint64_t)(uint32_t)outer[j]) * PRIME;
                decreasing |= (j > 0 && outer[j] < outer[j - 1]);
            }
            opart[c] = ho;
            bad[c] = (uint8_t)(out_of_range | (decreasing ? 1u : 0u));
        }
        uint64_t h = OFFSET ^ (uint64_t)n ^ ((uint64_t)nnz << 20);
        bool ok = outer[0] == 0 && (long long)outer[n] == nnz;
        for (int c = 0; c < chunks; ++c)
        {
            h = (h ^ opart[c]) * PRIME;
            h = (h ^ part[c]) * PRIME;
            ok = ok && !bad[c];
        }
        if (valid)
            *valid = ok;
        return h;
    }
} // namespace pmas
