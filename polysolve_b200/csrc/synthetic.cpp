// Seeded synthetic linear-elasticity systems on a structured tetrahedral mesh.
//
// This is the workload generator for the MAS-PCG solver: the unit cube is split into N^3
// cells, each cell into 6 tetrahedra along the main diagonal (Kuhn / Freudenthal split, so
// every vertex couples to 14 neighbours plus itself). The system is A = K + M / dt^2 with
// P1 linear-elasticity stiffness K (Lame parameters from E and nu per element) and a lumped
// mass M. Dirichlet vertices (the x = 0 face) become identity rows and columns, the same
// convention polysolve's dirichlet_solve uses (src/polysolve/linear/FEMSolver.cpp:106-153).
// Optional "contact" pairs add k n n^T couplings between nearby vertices.
//
// The matrix is emitted as scalar CSC (column-major, int32 indices, sorted rows), which is the
// layout of polysolve's StiffnessMatrix (src/polysolve/Types.hpp:11). A is exactly symmetric
// bit for bit, so the CSC arrays are also the CSR arrays of A.
//
// Randomness is counter based (splitmix64 of seed, stream and index), so the output does not
// depend on the thread count.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>

namespace
{
    inline uint64_t splitmix64(uint64_t x)
    {
        x += 0x9E3779B97F4A7C15ull;
        x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
        x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
        return x ^ (x >> 31);
    }

    // Uniform in (0, 1) from (seed, stream, index).
    inline double uniform01(uint64_t seed, uint64_t stream, uint64_t index)
    {
        uint64_t h = splitmix64(seed ^ splitmix64(stream * 0x632BE59BD9B4E019ull + index));
        return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }

    // Standard normal by Box-Muller from two counter draws.
    inline double normal01(uint64_t seed, uint64_t stream, uint64_t index)
    {
        double u1 = uniform01(seed, stream, 2 * index);
        double u2 = uniform01(seed, stream, 2 * index + 1);
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }

    enum Stream : uint64_t
    {
        STREAM_JITTER = 1,
        STREAM_YOUNG = 2,
        STREAM_CONTACT = 3,
        STREAM_PHASE = 4,
    };

    // The 15 stencil offsets of the Freudenthal triangulation: self, then the 7 positive
    // 0/1 offsets and their negatives. Slot order is fixed; columns are sorted later.
    const int STENCIL[15][3] = {
        {0, 0, 0},
        {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}, {1, 1, 1},
        {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}, {-1, -1, 0}, {0, -1, -1}, {-1, 0, -1}, {-1, -1, -1},
    };

    inline int stencil_slot(int dx, int dy, int dz)
    {
        for (int s = 0; s < 15; ++s)
            if (STENCIL[s][0] == dx && STENCIL[s][1] == dy && STENCIL[s][2] == dz)
                return s;
        return -1;
    }

    // Axis permutations: the 6 monotone paths from corner (0,0,0) to (1,1,1).
    const int PERMS[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

    struct Block
    {
        double a[9];
    };

    struct System
    {
        int n = 0;          // scalar dimension = 3 * nverts
        int nverts = 0;
        long long nnz = 0;
        std::vector<int> outer;
        std::vector<int> inner;
        std::vector<double> vals;
        std::vector<double> pos; // 3 * nverts
    };
} // namespace

extern "C"
{
    struct syn_params
    {
        int N;               // cells per edge
        double young;        // median Young's modulus
        double young_sigma;  // lognormal sigma of E per element (0 = constant)
        double poisson;
        double density;
        double dt;           // time step h in M / h^2
        double jitter;       // vertex jitter as a fraction of the grid spacing (0.2 = +-0.2 h)
        int dirichlet_x0;    // 1: fix the x = 0 face
        unsigned long long seed;
        int contact_pairs;   // number of random nearby vertex pairs with k n n^T couplings
        double contact_k;    // median contact stiffness
        double contact_sigma;
        const double *young_override; // optional per-element E (6 N^3 values), else NULL
    };

    void *syn_build(const syn_params *p);
    int syn_sizes(void *h, int *n, long long *nnz, int *nverts);
    int syn_copy(void *h, int *outer, int *inner, double *vals, double *pos);
    void syn_free(void *h);
    int syn_young(const syn_params *p, double *out);
}

namespace
{
    // Per-element Young's modulus exactly as syn_build draws it.
    inline double element_young(const syn_params &p, long long e)
    {
        if (p.young_override)
            return p.young_override[e];
        if (p.young_sigma <= 0.0)
            return p.young;
        return p.young * std::exp(p.young_sigma * normal01(p.seed, STREAM_YOUNG, (uint64_t)e));
    }
} // namespace

extern "C" int syn_young(const syn_params *p, double *out)
{
    const long long ne = 6LL * p->N * p->N * p->N;
#pragma omp parallel for schedule(static)
    for (long long e = 0; e < ne; ++e)
        out[e] = element_young(*p, e);
    return 0;
}

extern "C" void *syn_build(const syn_params *pp)
{
    const syn_params p = *pp;
    const int N = p.N;
    if (N < 1)
        return nullptr;
    const int M = N + 1;
    const int nv = M * M * M;
    const double h = 1.0 / N;
    auto vid = [M](int i, int j, int k) { return i + M * (j + M * k); };

    auto *sys = new System();
    sys->nverts = nv;
    sys->n = 3 * nv;
    sys->pos.resize(3 * (size_t)nv);

    // Vertex positions with jitter on the coordinates that are not on a cube face.
#pragma omp parallel for schedule(static)
    for (int v = 0; v < nv; ++v)
    {
        int idx[3] = {v % M, (v / M) % M, v / (M * M)};
        for (int d = 0; d < 3; ++d)
        {
            double x = idx[d] * h;
            if (p.jitter > 0.0 && idx[d] > 0 && idx[d] < N)
            {
                double u = uniform01(p.seed, STREAM_JITTER, 3ull * v + d);
                x += (2.0 * u - 1.0) * p.jitter * h;
            }
            sys->pos[3 * (size_t)v + d] = x;
        }
    }

    // Stencil blocks: 15 slots per vertex.
    std::vector<Block> blocks((size_t)nv * 15);
    std::memset(blocks.data(), 0, blocks.size() * sizeof(Block));

    const double nu = p.poisson;

    // Assemble by 8 colours of cells (i, j, k parity): cells of one colour share no vertex.
    for (int color = 0; color < 8; ++color)
    {
        const int ci = color & 1, cj = (color >> 1) & 1, ck = (color >> 2) & 1;
        const int ni = (N - ci + 1) / 2, nj = (N - cj + 1) / 2, nk = (N - ck + 1) / 2;
        const long long ncells = (long long)ni * nj * nk;
#pragma omp parallel for schedule(static)
        for (long long c = 0; c < ncells; ++c)
        {
            const int i = ci + 2 * (int)(c % ni);
            const int j = cj + 2 * (int)((c / ni) % nj);
            const int k = ck + 2 * (int)(c / ((long long)ni * nj));
            const long long cell = i + (long long)N * (j + (long long)N * k);
            for (int t = 0; t < 6; ++t)
            {
                int off[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {1, 1, 1}};
                off[1][PERMS[t][0]] = 1;
                for (int d = 0; d < 3; ++d)
                    off[2][d] = off[1][d];
                off[2][PERMS[t][1]] = 1;
                int vv[4];
                double X[4][3];
                for (int a = 0; a < 4; ++a)
                {
                    vv[a] = vid(i + off[a][0], j + off[a][1], k + off[a][2]);
                    for (int d = 0; d < 3; ++d)
                        X[a][d] = sys->pos[3 * (size_t)vv[a] + d];
                }
                // Jacobian columns x_a - x_0.
                double J[3][3];
                for (int d = 0; d < 3; ++d)
                    for (int a = 0; a < 3; ++a)
                        J[d][a] = X[a + 1][d] - X[0][d];
                double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1])
                             - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0])
                             + J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
                double inv[3][3];
                inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
                inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
                inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
                inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
                inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
                inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
                inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
                inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
                inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
                const double vol = std::fabs(det) / 6.0;
                // Shape gradients: rows of J^-1 for nodes 1..3, node 0 is minus their sum.
                double g[4][3];
                for (int d = 0; d < 3; ++d)
                {
                    g[1][d] = inv[0][d];
                    g[2][d] = inv[1][d];
                    g[3][d] = inv[2][d];
                    g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
                }
                const double E = element_young(p, cell * 6 + t);
                const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
                const double mu = E / (2.0 * (1.0 + nu));
                const double lumped = p.density * vol / 4.0 / (p.dt * p.dt);
                for (int a = 0; a < 4; ++a)
                {
                    for (int b = a; b < 4; ++b)
                    {
                        double gab = g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2];
                        double Kab[9];
                        for (int r = 0; r < 3; ++r)
                            for (int s = 0; s < 3; ++s)
                                Kab[3 * r + s] = vol * (lam * g[a][r] * g[b][s] + mu * g[b][r] * g[a][s]
                                                        + (r == s ? mu * gab : 0.0));
                        if (a == b)
                        {
                            // Symmetrise the diagonal block exactly, then add the lumped mass.
                            for (int r = 0; r < 3; ++r)
                                for (int s = r + 1; s < 3; ++s)
                                    Kab[3 * s + r] = Kab[3 * r + s];
                            for (int r = 0; r < 3; ++r)
                                Kab[4 * r] += lumped;
                            Block &B = blocks[(size_t)vv[a] * 15];
                            for (int q = 0; q < 9; ++q)
                                B.a[q] += Kab[q];
                        }
                        else
                        {
                            const int sa = (vv[b] % M) - (vv[a] % M), sb = ((vv[b] / M) % M) - ((vv[a] / M) % M),
                                      sc = (vv[b] / (M * M)) - (vv[a] / (M * M));
                            const int slot_ab = stencil_slot(sa, sb, sc);
                            const int slot_ba = stencil_slot(-sa, -sb, -sc);
                            Block &Bab = blocks[(size_t)vv[a] * 15 + slot_ab];
                            Block &Bba = blocks[(size_t)vv[b] * 15 + slot_ba];
                            for (int r = 0; r < 3; ++r)
                                for (int s = 0; s < 3; ++s)
                                {
                                    Bab.a[3 * r + s] += Kab[3 * r + s];
                                    Bba.a[3 * s + r] += Kab[3 * r + s];
                                }
                        }
                    }
                }
            }
        }
    }

    // Contact pairs: extra blocks, kept per vertex in sorted lists.
    std::vector<std::vector<std::pair<int, Block>>> extra(p.contact_pairs > 0 ? nv : 0);
    std::vector<Block> extra_diag;
    if (p.contact_pairs > 0)
    {
        extra_diag.assign(nv, Block{});
        // Candidate offsets within two grid steps.
        std::vector<std::array<int, 3>> cand;
        for (int dz = -2; dz <= 2; ++dz)
            for (int dy = -2; dy <= 2; ++dy)
                for (int dx = -2; dx <= 2; ++dx)
                    if (dx || dy || dz)
                        cand.push_back({dx, dy, dz});
        long long drawn = 0;
        int made = 0;
        while (made < p.contact_pairs && drawn < 1000LL * p.contact_pairs)
        {
            const uint64_t base = (uint64_t)drawn;
            ++drawn;
            int v = (int)(uniform01(p.seed, STREAM_CONTACT, 4 * base) * nv);
            v = std::min(v, nv - 1);
            int ci2 = (int)(uniform01(p.seed, STREAM_CONTACT, 4 * base + 1) * cand.size());
            ci2 = std::min<int>(ci2, (int)cand.size() - 1);
            int i = v % M + cand[ci2][0], j = (v / M) % M + cand[ci2][1], k = v / (M * M) + cand[ci2][2];
            if (i < 0 || j < 0 || k < 0 || i > N || j > N || k > N)
                continue;
            int w = vid(i, j, k);
            double d[3], len2 = 0.0;
            for (int q = 0; q < 3; ++q)
            {
                d[q] = sys->pos[3 * (size_t)w + q] - sys->pos[3 * (size_t)v + q];
                len2 += d[q] * d[q];
            }
            if (len2 >= 4.0 * h * h || len2 <= 0.0)
                continue;
            double len = std::sqrt(len2);
            for (int q = 0; q < 3; ++q)
                d[q] /= len;
            double kk = p.contact_k * std::exp(p.contact_sigma * normal01(p.seed, STREAM_CONTACT, 4 * base + 2));
            Block nn;
            for (int r = 0; r < 3; ++r)
                for (int s = r; s < 3; ++s)
                    nn.a[3 * r + s] = nn.a[3 * s + r] = kk * d[r] * d[s];
            for (int q = 0; q < 9; ++q)
            {
                extra_diag[v].a[q] += nn.a[q];
                extra_diag[w].a[q] += nn.a[q];
            }
            Block neg;
            for (int q = 0; q < 9; ++q)
                neg.a[q] = -nn.a[q];
            auto add_off = [&](int row, int col) {
                auto &lst = extra[row];
                for (auto &e : lst)
                    if (e.first == col)
                    {
                        for (int q = 0; q < 9; ++q)
                            e.second.a[q] += neg.a[q];
                        return;
                    }
                lst.push_back({col, neg});
            };
            add_off(v, w);
            add_off(w, v);
            ++made;
        }
    }

    auto fixed = [&](int v) { return p.dirichlet_x0 && (v % M) == 0; };

    // Scalar entries per scalar row of each vertex, then the emitted rows.
    std::vector<long long> row_nnz(nv, 0);
#pragma omp parallel for schedule(static)
    for (int v = 0; v < nv; ++v)
    {
        if (fixed(v))
        {
            row_nnz[v] = 1; // per scalar row: just the diagonal
            continue;
        }
        const int i = v % M, j = (v / M) % M, k = v / (M * M);
        std::vector<int> cols;
        for (int s = 0; s < 15; ++s)
        {
            int a = i + STENCIL[s][0], b = j + STENCIL[s][1], c = k + STENCIL[s][2];
            if (a < 0 || b < 0 || c < 0 || a > N || b > N || c > N)
                continue;
            int w = vid(a, b, c);
            if (w != v && fixed(w))
                continue;
            cols.push_back(w);
        }
        if (p.contact_pairs > 0)
            for (auto &e : extra[v])
                if (!fixed(e.first) && std::find(cols.begin(), cols.end(), e.first) == cols.end())
                    cols.push_back(e.first);
        row_nnz[v] = 3LL * (long long)cols.size();
    }
    std::vector<long long> row_off(nv + 1, 0);
    for (int v = 0; v < nv; ++v)
        row_off[v + 1] = row_off[v] + 3 * row_nnz[v];
    const long long nnz = row_off[nv];
    sys->nnz = nnz;
    sys->outer.resize((size_t)sys->n + 1);
    sys->inner.resize((size_t)nnz);
    sys->vals.resize((size_t)nnz);

#pragma omp parallel for schedule(dynamic, 256)
    for (int v = 0; v < nv; ++v)
    {
        long long o = row_off[v];
        if (fixed(v))
        {
            for (int r = 0; r < 3; ++r)
            {
                sys->outer[3 * (size_t)v + r] = (int)(o + r);
                sys->inner[o + r] = 3 * v + r;
                sys->vals[o + r] = 1.0;
            }
            continue;
        }
        const int i = v % M, j = (v / M) % M, k = v / (M * M);
        std::vector<std::pair<int, Block>> cols;
        for (int s = 0; s < 15; ++s)
        {
            int a = i + STENCIL[s][0], b = j + STENCIL[s][1], c = k + STENCIL[s][2];
            if (a < 0 || b < 0 || c < 0 || a > N || b > N || c > N)
                continue;
            int w = vid(a, b, c);
            if (w != v && fixed(w))
                continue;
            Block B = blocks[(size_t)v * 15 + s];
            if (s == 0 && p.contact_pairs > 0)
                for (int q = 0; q < 9; ++q)
                    B.a[q] += extra_diag[v].a[q];
            cols.push_back({w, B});
        }
        if (p.contact_pairs > 0)
            for (auto &e : extra[v])
            {
                if (fixed(e.first))
                    continue;
                bool merged = false;
                for (auto &c : cols)
                    if (c.first == e.first)
                    {
                        for (int q = 0; q < 9; ++q)
                            c.second.a[q] += e.second.a[q];
                        merged = true;
                        break;
                    }
                if (!merged)
                    cols.push_back(e);
            }
        std::sort(cols.begin(), cols.end(), [](const auto &x, const auto &y) { return x.first < y.first; });
        const int cnt = (int)cols.size();
        for (int r = 0; r < 3; ++r)
        {
            long long ro = o + (long long)r * 3 * cnt;
            sys->outer[3 * (size_t)v + r] = (int)ro;
            for (int c = 0; c < cnt; ++c)
                for (int s = 0; s < 3; ++s)
                {
                    sys->inner[ro + 3 * c + s] = 3 * cols[c].first + s;
                    sys->vals[ro + 3 * c + s] = cols[c].second.a[3 * r + s];
                }
        }
    }
    sys->outer[sys->n] = (int)nnz;
    return sys;
}

extern "C" int syn_sizes(void *h, int *n, long long *nnz, int *nverts)
{
    auto *s = static_cast<System *>(h);
    if (!s)
        return 1;
    *n = s->n;
    *nnz = s->nnz;
    *nverts = s->nverts;
    return 0;
}

extern "C" int syn_copy(void *h, int *outer, int *inner, double *vals, double *pos)
{
    auto *s = static_cast<System *>(h);
    if (!s)
        return 1;
    if (outer)
        std::memcpy(outer, s->outer.data(), s->outer.size() * sizeof(int));
    if (inner)
        std::memcpy(inner, s->inner.data(), s->inner.size() * sizeof(int));
    if (vals)
        std::memcpy(vals, s->vals.data(), s->vals.size() * sizeof(double));
    if (pos)
        std::memcpy(pos, s->pos.data(), s->pos.size() * sizeof(double));
    return 0;
}

extern "C" void syn_free(void *h)
{
    delete static_cast<System *>(h);
}
