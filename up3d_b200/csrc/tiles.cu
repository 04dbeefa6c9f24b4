// Tile plan of the tiled residual + Jacobian assembly (tiles.cuh): built
// on the host once per mesh and tile size, checked, then uploaded.
//
//   1. connected components of the face graph (union-find), so that cases
//      concatenated into one mesh are tiled one by one, exactly as each
//      case alone;
//   2. per component, recursive coordinate bisection of the element
//      centroids: split along the longest extent of the bounding box at a
//      multiple of T elements (ties by user id), down to tiles of T; the
//      elements of a tile in ascending user id;
//   3. per tile (OpenMP): its distinct nodes, the local connectivity, the
//      incident entries of every node and the contributors of every
//      element edge, both in ascending local element;
//   4. ownership: a node output belongs to the tile when the tile holds
//      all of the node's incident elements, an upper slot when it holds all
//      elements containing the edge; the rest get partial-sum positions,
//      numbered tile by tile, and combine lists in tile order.

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "tiles.cuh"

namespace up3d {

namespace {

struct Dsu {
    std::vector<int32_t> p;
    explicit Dsu(int64_t n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int32_t find(int32_t x) {
        while (p[x] != x) {
            p[x] = p[p[x]];
            x = p[x];
        }
        return x;
    }
    void unite(int32_t a, int32_t b) {
        a = find(a);
        b = find(b);
        if (a == b) return;
        if (a < b) std::swap(a, b);
        p[a] = b;  // the smaller id is the root
    }
};

// Recursive coordinate bisection of a[0, n) into runs of T (all full but
// the last); a holds user element ids.
void rcb(int32_t* a, int64_t n, int T, const std::vector<double4>& cen, double stretch, int depth) {
    if (n <= T) {
        std::sort(a, a + n);
        return;
    }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t k = 0; k < n; ++k) {
        const double4 c = cen[a[k]];
        lo[0] = std::min(lo[0], c.x); hi[0] = std::max(hi[0], c.x);
        lo[1] = std::min(lo[1], c.y); hi[1] = std::max(hi[1], c.y);
        lo[2] = std::min(lo[2], c.z); hi[2] = std::max(hi[2], c.z);
    }
    // the longest extent, x counted 1/stretch: tiles `stretch` times longer
    // along x than across
    const double ext[3] = {(hi[0] - lo[0]) / stretch, hi[1] - lo[1], hi[2] - lo[2]};
    int ax = 0;
    for (int d = 1; d < 3; ++d)
        if (ext[d] > ext[ax]) ax = d;
    const int64_t nt = (n + T - 1) / T;
    const int64_t k = (nt / 2) * T;
    auto coord = [&](int32_t e) {
        const double4 c = cen[e];
        return ax == 0 ? c.x : (ax == 1 ? c.y : c.z);
    };
    std::nth_element(a, a + k, a + n, [&](int32_t x, int32_t y) {
        const double cx = coord(x), cy = coord(y);
        return cx < cy || (cx == cy && x < y);
    });
    if (depth < 6 && n > 65536) {
#pragma omp task shared(cen)
        rcb(a, k, T, cen, stretch, depth + 1);
#pragma omp task shared(cen)
        rcb(a + k, n - k, T, cen, stretch, depth + 1);
#pragma omp taskwait
    } else {
        rcb(a, k, T, cen, stretch, depth + 1);
        rcb(a + k, n - k, T, cen, stretch, depth + 1);
    }
}

struct TileHost {
    std::vector<int32_t> nodes;                   // distinct global nodes, ascending
    std::vector<int32_t> nent_off;                // (nodes + 1)
    std::vector<uint16_t> nent;
    std::vector<int32_t> eslot;                   // the upper slot of each distinct edge
    std::vector<int32_t> uent_off;                // (edges + 1)
    std::vector<uint16_t> uent;
};

constexpr int PAIR_I[6] = {0, 0, 0, 1, 1, 2};
constexpr int PAIR_J[6] = {1, 2, 3, 2, 3, 3};

}  // namespace

// The plan as host arrays (uploaded as they are into a TilePlan).
struct PlanHost {
    int32_t T = 0, stretch = 1, max_nodes = 0, max_edges = 0;
    int64_t n_tiles = 0, n_tile_nodes = 0, n_tile_edges = 0, n_part = 0;
    std::vector<int32_t> perm, iperm, eoff, noff, uoff, tnode, nent_off, uent_off;
    std::vector<ushort4> lconn;
    std::vector<uint16_t> nent, uent;
    std::vector<int2> ndst, udst, cn_dst, ce_dst;
    std::vector<int32_t> cn_off, cn_idx, ce_off, ce_idx;
    std::vector<int4> conn_t, fn_t;
    std::vector<double4> cen_t;
};

// Builds the plan from host copies of the mesh data: connectivity, face
// neighbours, centroids and the P1 pattern (sorted rows).
PlanHost build_plan_host(const std::vector<int4>& conn, const std::vector<int4>& fn, const std::vector<double4>& cen,
                         int64_t N, const std::vector<int32_t>& indptr, const std::vector<int32_t>& indices,
                         int T, int stretch) {
    UP3D_REQUIRE(T == 128 || T == 256, UP3D_ERR_VALUE, "tile plan: tile_elems must be 128 or 256");
    UP3D_REQUIRE(stretch == 1 || stretch == 2 || stretch == 4, UP3D_ERR_VALUE,
                 "tile plan: tile_stretch must be 1, 2 or 4");
    const int64_t E = (int64_t)conn.size(), Z = (int64_t)indices.size();
    // absolute diagonal slot of each row (-1 for an empty row) and the
    // transposed slot of every entry
    auto find = [&](int32_t r, int32_t c) -> int32_t {
        const int32_t* b = indices.data() + indptr[r];
        const int32_t* e = indices.data() + indptr[r + 1];
        const int32_t* f = std::lower_bound(b, e, c);
        return (f == e || *f != c) ? -1 : (int32_t)(f - indices.data());
    };
    std::vector<int32_t> diag(N), zt(Z);
    int bad_pattern = 0;
#pragma omp parallel for schedule(static) reduction(| : bad_pattern)
    for (int64_t r = 0; r < N; ++r) {
        diag[r] = find((int32_t)r, (int32_t)r);
        for (int32_t k = indptr[r]; k < indptr[r + 1]; ++k) {
            zt[k] = find(indices[k], (int32_t)r);
            if (zt[k] < 0) bad_pattern = 1;
        }
    }
    UP3D_REQUIRE(!bad_pattern, UP3D_ERR_VALUE, "tile plan: the pattern is not structurally symmetric");

    // ---- 1. components of the face graph, in order of their smallest element
    Dsu dsu(E);
    for (int64_t e = 0; e < E; ++e) {
        const int nb[4] = {fn[e].x, fn[e].y, fn[e].z, fn[e].w};
        for (int k = 0; k < 4; ++k)
            if (nb[k] >= 0 && nb[k] < E) dsu.unite((int32_t)e, nb[k]);
    }
    std::vector<int32_t> root(E);
    for (int64_t e = 0; e < E; ++e) root[e] = dsu.find((int32_t)e);
    std::vector<int32_t> comp_id(E, -1);
    int32_t n_comp = 0;
    for (int64_t e = 0; e < E; ++e)
        if (root[e] == e) comp_id[e] = n_comp++;
    std::vector<int64_t> comp_off(n_comp + 1, 0);
    for (int64_t e = 0; e < E; ++e) comp_off[comp_id[root[e]] + 1]++;
    for (int32_t c = 0; c < n_comp; ++c) comp_off[c + 1] += comp_off[c];
    std::vector<int32_t> order(E);
    {
        std::vector<int64_t> cur(comp_off.begin(), comp_off.end() - 1);
        for (int64_t e = 0; e < E; ++e) order[cur[comp_id[root[e]]]++] = (int32_t)e;
    }
    // ---- 2. bisection per component; tiles of T within each component
#pragma omp parallel
#pragma omp single
    for (int32_t c = 0; c < n_comp; ++c)
        rcb(order.data() + comp_off[c], comp_off[c + 1] - comp_off[c], T, cen, (double)stretch, 0);
    std::vector<int32_t> eoff(1, 0);
    for (int32_t c = 0; c < n_comp; ++c)
        for (int64_t b = comp_off[c]; b < comp_off[c + 1]; b += T)
            eoff.push_back((int32_t)std::min<int64_t>(b + T, comp_off[c + 1]));
    const int64_t n_tiles = (int64_t)eoff.size() - 1;
    std::vector<int32_t> iperm(E);
    for (int64_t x = 0; x < E; ++x) iperm[order[x]] = (int32_t)x;

    // ---- 3. per tile: nodes, local connectivity, node entries, edges
    std::vector<TileHost> th(n_tiles);
    std::vector<ushort4> lconn(E);
    int bad_slot = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : bad_slot)
    for (int64_t t = 0; t < n_tiles; ++t) {
        TileHost& h = th[t];
        const int32_t e0 = eoff[t], ne = eoff[t + 1] - e0;
        h.nodes.resize(4 * (size_t)ne);
        for (int32_t l = 0; l < ne; ++l) {
            const int4 c = conn[order[e0 + l]];
            h.nodes[4 * l] = c.x;
            h.nodes[4 * l + 1] = c.y;
            h.nodes[4 * l + 2] = c.z;
            h.nodes[4 * l + 3] = c.w;
        }
        std::sort(h.nodes.begin(), h.nodes.end());
        h.nodes.erase(std::unique(h.nodes.begin(), h.nodes.end()), h.nodes.end());
        const int32_t nn = (int32_t)h.nodes.size();
        auto lidx = [&](int32_t g) {
            return (uint16_t)(std::lower_bound(h.nodes.begin(), h.nodes.end(), g) - h.nodes.begin());
        };
        std::vector<uint16_t> lc(4 * (size_t)ne);
        for (int32_t l = 0; l < ne; ++l) {
            const int4 c = conn[order[e0 + l]];
            lc[4 * l] = lidx(c.x);
            lc[4 * l + 1] = lidx(c.y);
            lc[4 * l + 2] = lidx(c.z);
            lc[4 * l + 3] = lidx(c.w);
            lconn[e0 + l] = make_ushort4(lc[4 * l], lc[4 * l + 1], lc[4 * l + 2], lc[4 * l + 3]);
        }
        // node entries, ascending local element (counting sort)
        h.nent_off.assign(nn + 1, 0);
        for (size_t k = 0; k < lc.size(); ++k) h.nent_off[lc[k] + 1]++;
        for (int32_t r = 0; r < nn; ++r) h.nent_off[r + 1] += h.nent_off[r];
        h.nent.resize(4 * (size_t)ne);
        {
            std::vector<int32_t> cur(h.nent_off.begin(), h.nent_off.end() - 1);
            for (int32_t l = 0; l < ne; ++l)
                for (int i = 0; i < 4; ++i) h.nent[cur[lc[4 * l + i]]++] = (uint16_t)((l << 2) | i);
        }
        // edges: (key, code) in local element order, stably grouped by key
        std::vector<std::pair<int64_t, uint16_t>> pr(6 * (size_t)ne);
        for (int32_t l = 0; l < ne; ++l) {
            const int4 c = conn[order[e0 + l]];
            const int32_t v[4] = {c.x, c.y, c.z, c.w};
            for (int p = 0; p < 6; ++p) {
                const int64_t a = v[PAIR_I[p]], b = v[PAIR_J[p]];
                pr[6 * l + p] = {(std::min(a, b) << 32) | std::max(a, b), (uint16_t)((l << 3) | p)};
            }
        }
        std::stable_sort(pr.begin(), pr.end(),
                         [](const std::pair<int64_t, uint16_t>& x, const std::pair<int64_t, uint16_t>& y) {
                             return x.first < y.first;
                         });
        h.uent.resize(pr.size());
        for (size_t k = 0; k < pr.size(); ++k) {
            if (k == 0 || pr[k].first != pr[k - 1].first) {
                h.uent_off.push_back((int32_t)k);
                const int32_t r = (int32_t)(pr[k].first >> 32), col = (int32_t)(pr[k].first & 0xFFFFFFFF);
                const int32_t* b = indices.data() + indptr[r];
                const int32_t* e = indices.data() + indptr[r + 1];
                const int32_t* f = std::lower_bound(b, e, col);
                if (f == e || *f != col) {
                    bad_slot = 1;
                    h.eslot.push_back(0);
                } else {
                    h.eslot.push_back((int32_t)(f - indices.data()));
                }
            }
            h.uent[k] = pr[k].second;
        }
        h.uent_off.push_back((int32_t)pr.size());
    }
    UP3D_REQUIRE(!bad_slot, UP3D_ERR_RUNTIME, "tile plan: an element edge is missing from the P1 pattern");

    // ---- 4. ownership, partial numbering and the combine lists
    std::vector<int32_t> deg(N, 0);
    for (int64_t e = 0; e < E; ++e) {
        deg[conn[e].x]++;
        deg[conn[e].y]++;
        deg[conn[e].z]++;
        deg[conn[e].w]++;
    }
    std::vector<int32_t> ecnt(Z, 0);
    for (int64_t t = 0; t < n_tiles; ++t) {
        const TileHost& h = th[t];
        for (size_t q = 0; q < h.eslot.size(); ++q) ecnt[h.eslot[q]] += h.uent_off[q + 1] - h.uent_off[q];
    }
    std::vector<int32_t> noff(n_tiles + 1, 0), uoff(n_tiles + 1, 0);
    for (int64_t t = 0; t < n_tiles; ++t) {
        noff[t + 1] = noff[t] + (int32_t)th[t].nodes.size();
        uoff[t + 1] = uoff[t] + (int32_t)th[t].eslot.size();
    }
    const int64_t n_tn = noff[n_tiles], n_te = uoff[n_tiles];
    std::vector<int32_t> tnode(n_tn), nent_off(n_tn + 1), uent_off(n_te + 1), tedge_slot(n_te);
    std::vector<uint16_t> nent(4 * (size_t)E), uent(6 * (size_t)E);
    std::vector<int2> ndst(n_tn), udst(n_te);
    std::vector<int32_t> node_pc(N + 1, 0), slot_pc(Z + 1, 0);  // partials per node / slot
    int64_t q = 0;
    int32_t max_nodes = 0, max_edges = 0;
    {
        int64_t ne_run = 0, ue_run = 0;
        for (int64_t t = 0; t < n_tiles; ++t) {
            const TileHost& h = th[t];
            max_nodes = std::max<int32_t>(max_nodes, (int32_t)h.nodes.size());
            max_edges = std::max<int32_t>(max_edges, (int32_t)h.eslot.size());
            for (size_t r = 0; r < h.nodes.size(); ++r) {
                const int64_t p = noff[t] + (int64_t)r;
                const int32_t n = h.nodes[r];
                tnode[p] = n;
                nent_off[p] = (int32_t)(ne_run + h.nent_off[r]);
                const int32_t cnt = h.nent_off[r + 1] - h.nent_off[r];
                if (cnt == deg[n]) {
                    ndst[p] = make_int2(n, diag[n]);
                } else {
                    ndst[p] = make_int2((int32_t)(-1 - q), diag[n]);
                    node_pc[n + 1]++;
                    q += 2;
                }
            }
            std::memcpy(nent.data() + ne_run, h.nent.data(), sizeof(uint16_t) * h.nent.size());
            ne_run += (int64_t)h.nent.size();
            for (size_t k = 0; k < h.eslot.size(); ++k) {
                const int64_t p = uoff[t] + (int64_t)k;
                const int32_t sl = h.eslot[k];
                tedge_slot[p] = sl;
                uent_off[p] = (int32_t)(ue_run + h.uent_off[k]);
                const int32_t cnt = h.uent_off[k + 1] - h.uent_off[k];
                if (cnt == ecnt[sl]) {
                    udst[p] = make_int2(sl, zt[sl]);
                } else {
                    udst[p] = make_int2((int32_t)(-1 - q), 0);
                    slot_pc[sl + 1]++;
                    q += 1;
                }
            }
            std::memcpy(uent.data() + ue_run, h.uent.data(), sizeof(uint16_t) * h.uent.size());
            ue_run += (int64_t)h.uent.size();
        }
        nent_off[n_tn] = (int32_t)ne_run;
        uent_off[n_te] = (int32_t)ue_run;
    }
    UP3D_REQUIRE(q < (1ll << 31), UP3D_ERR_VALUE, "tile plan: too many partial sums");
    th.clear();
    th.shrink_to_fit();
    // combine lists: split nodes and isolated nodes (R = 0), split slots;
    // partial positions in tile order
    std::vector<int32_t> cn_off(1, 0), cn_idx;
    std::vector<int2> cn_dst;
    std::vector<int32_t> ce_off(1, 0), ce_idx;
    std::vector<int2> ce_dst;
    {
        std::vector<int32_t> nfirst(N + 1, 0), sfirst(Z + 1, 0);
        for (int64_t n = 0; n < N; ++n) nfirst[n + 1] = nfirst[n] + node_pc[n + 1];
        for (int64_t z = 0; z < Z; ++z) sfirst[z + 1] = sfirst[z] + slot_pc[z + 1];
        std::vector<int32_t> nlist(nfirst[N]), slist(sfirst[Z]);
        std::vector<int32_t> ncur(nfirst.begin(), nfirst.end() - 1), scur(sfirst.begin(), sfirst.end() - 1);
        for (int64_t p = 0; p < n_tn; ++p)  // tile-major: tile order within each node
            if (ndst[p].x < 0) nlist[ncur[tnode[p]]++] = -1 - ndst[p].x;
        for (int64_t p = 0; p < n_te; ++p)
            if (udst[p].x < 0) slist[scur[tedge_slot[p]]++] = -1 - udst[p].x;
        for (int64_t n = 0; n < N; ++n) {
            if (nfirst[n + 1] == nfirst[n] && deg[n] > 0) continue;  // owned by one tile
            for (int32_t j = nfirst[n]; j < nfirst[n + 1]; ++j) cn_idx.push_back(nlist[j]);
            cn_off.push_back((int32_t)cn_idx.size());
            cn_dst.push_back(make_int2((int32_t)n, deg[n] > 0 ? diag[n] : -1));
        }
        for (int64_t z = 0; z < Z; ++z) {
            if (sfirst[z + 1] == sfirst[z]) continue;
            for (int32_t j = sfirst[z]; j < sfirst[z + 1]; ++j) ce_idx.push_back(slist[j]);
            ce_off.push_back((int32_t)ce_idx.size());
            ce_dst.push_back(make_int2((int32_t)z, zt[z]));
        }
    }
    // consistency of the plan before anything reads through it: every local
    // index inside its tile, every destination inside its array
    {
        int bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : bad)
        for (int64_t t = 0; t < n_tiles; ++t) {
            const int32_t ne = eoff[t + 1] - eoff[t], nn = noff[t + 1] - noff[t];
            if (ne <= 0 || ne > T || nn <= 0 || nn > 4 * T) bad |= 1;
            for (int32_t x = eoff[t]; x < eoff[t + 1]; ++x) {
                const ushort4 l = lconn[x];
                if (l.x >= nn || l.y >= nn || l.z >= nn || l.w >= nn) bad |= 2;
            }
            for (int32_t p = noff[t]; p < noff[t + 1]; ++p) {
                for (int32_t k = nent_off[p]; k < nent_off[p + 1]; ++k)
                    if ((nent[k] >> 2) >= ne) bad |= 4;
                const int2 d = ndst[p];
                if (d.x >= 0 ? (d.x >= N || d.y < 0 || d.y >= Z) : (-1ll - d.x + 1 >= q)) bad |= 8;
            }
            for (int32_t p = uoff[t]; p < uoff[t + 1]; ++p) {
                for (int32_t k = uent_off[p]; k < uent_off[p + 1]; ++k)
                    if ((uent[k] >> 3) >= ne || (uent[k] & 7) >= 6) bad |= 16;
                const int2 d = udst[p];
                if (d.x >= 0 ? (d.x >= Z || d.y < 0 || d.y >= Z) : (-1ll - d.x >= q)) bad |= 32;
            }
        }
        for (size_t k = 0; k < cn_idx.size(); ++k)
            if (cn_idx[k] < 0 || (int64_t)cn_idx[k] + 1 >= q) bad |= 64;
        for (size_t k = 0; k < ce_idx.size(); ++k)
            if (ce_idx[k] < 0 || ce_idx[k] >= q) bad |= 64;
        for (const int2& d : cn_dst)
            if (d.x < 0 || d.x >= N || d.y >= Z) bad |= 128;
        for (const int2& d : ce_dst)
            if (d.x < 0 || d.x >= Z || d.y < 0 || d.y >= Z) bad |= 128;
        UP3D_REQUIRE(!bad, UP3D_ERR_RUNTIME, "tile plan: inconsistent plan (code " + std::to_string(bad) + ")");
        UP3D_REQUIRE(nent_off[n_tn] == 4 * E && uent_off[n_te] == 6 * E, UP3D_ERR_RUNTIME,
                     "tile plan: entry counts do not cover the mesh");
    }
    // internal-order copies of the element data
    std::vector<int4> conn_t(E), fn_t(E);
    std::vector<double4> cen_t(E);
#pragma omp parallel for schedule(static)
    for (int64_t x = 0; x < E; ++x) {
        const int32_t e = order[x];
        conn_t[x] = conn[e];
        cen_t[x] = cen[e];
        int nb[4] = {fn[e].x, fn[e].y, fn[e].z, fn[e].w};
        for (int k = 0; k < 4; ++k) nb[k] = (nb[k] >= 0 && nb[k] < E) ? iperm[nb[k]] : -1;
        fn_t[x] = make_int4(nb[0], nb[1], nb[2], nb[3]);
    }

    PlanHost H;
    H.T = T;
    H.stretch = stretch;
    H.max_nodes = max_nodes;
    H.max_edges = max_edges;
    H.n_tiles = n_tiles;
    H.n_tile_nodes = n_tn;
    H.n_tile_edges = n_te;
    H.n_part = q;
    H.perm = std::move(order);
    H.iperm = std::move(iperm);
    H.eoff = std::move(eoff);
    H.noff = std::move(noff);
    H.uoff = std::move(uoff);
    H.tnode = std::move(tnode);
    H.lconn = std::move(lconn);
    H.nent_off = std::move(nent_off);
    H.nent = std::move(nent);
    H.ndst = std::move(ndst);
    H.uent_off = std::move(uent_off);
    H.uent = std::move(uent);
    H.udst = std::move(udst);
    H.cn_off = std::move(cn_off);
    H.cn_idx = std::move(cn_idx);
    H.cn_dst = std::move(cn_dst);
    H.ce_off = std::move(ce_off);
    H.ce_idx = std::move(ce_idx);
    H.ce_dst = std::move(ce_dst);
    H.conn_t = std::move(conn_t);
    H.fn_t = std::move(fn_t);
    H.cen_t = std::move(cen_t);
    return H;
}

namespace {
// tile-node positions in plan order (the kernel stages them with one
// coalesced copy per tile)
__global__ void k_tile_xyz(int64_t n, const int32_t* __restrict__ tnode, const double4* __restrict__ X,
                           double4* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = X[tnode[i]];
}
// the mesh's face-displacement records in internal order
__global__ void k_tile_disp(int64_t E, const int32_t* __restrict__ perm, const double* __restrict__ disp,
                            double* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < 12 * E;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = disp[12 * (int64_t)perm[i / 12] + i % 12];
}
}  // namespace

void ensure_tiles(up3d_mesh* m, int T, int stretch, cudaStream_t s) {
    if (m->tiles && m->tiles->T == T && m->tiles->stretch == stretch) return;
    UP3D_REQUIRE(T == 128 || T == 256, UP3D_ERR_VALUE, "tile plan: tile_elems must be 128 or 256");
    const auto t_start = std::chrono::steady_clock::now();
    const int64_t E = m->E, N = m->N, Z = m->nnz;
    // host copies of the mesh data the plan needs
    std::vector<int4> conn(E), fn(E);
    std::vector<double4> cen(E);
    std::vector<int32_t> indptr(N + 1), indices(Z);
    UP3D_CUDA(cudaMemcpyAsync(conn.data(), m->conn.get(), sizeof(int4) * E, cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaMemcpyAsync(fn.data(), m->fnbr.get(), sizeof(int4) * E, cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaMemcpyAsync(cen.data(), m->cen.get(), sizeof(double4) * E, cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaMemcpyAsync(indptr.data(), m->indptr.get(), sizeof(int32_t) * (N + 1), cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaMemcpyAsync(indices.data(), m->indices.get(), sizeof(int32_t) * Z, cudaMemcpyDeviceToHost, s));
    UP3D_CUDA(cudaStreamSynchronize(s));
    PlanHost H = build_plan_host(conn, fn, cen, N, indptr, indices, T, stretch);
    auto P = std::make_shared<TilePlan>();
    P->T = T;
    P->stretch = stretch;
    P->max_edges = H.max_edges;
    P->n_tiles = H.n_tiles;
    P->max_nodes = H.max_nodes;
    P->n_tile_nodes = H.n_tile_nodes;
    P->n_tile_edges = H.n_tile_edges;
    P->n_part = H.n_part;
    P->n_cnode = (int64_t)H.cn_dst.size();
    P->n_cedge = (int64_t)H.ce_dst.size();
    // 16 bytes of padding after every array: the kernel stages a tile's
    // ranges in whole 16-byte blocks
    auto up = [&](auto& buf, const auto& vec) {
        buf.alloc(vec.size() + 16 / sizeof(vec[0]) + 1);
        if (!vec.empty())
            UP3D_CUDA(cudaMemcpyAsync(buf.get(), vec.data(), sizeof(vec[0]) * vec.size(), cudaMemcpyHostToDevice, s));
    };
    up(P->perm, H.perm);
    up(P->iperm, H.iperm);
    up(P->conn, H.conn_t);
    up(P->fnbr, H.fn_t);
    up(P->cen, H.cen_t);
    up(P->eoff, H.eoff);
    up(P->noff, H.noff);
    up(P->uoff, H.uoff);
    up(P->tnode, H.tnode);
    up(P->lconn, H.lconn);
    up(P->nent_off, H.nent_off);
    up(P->nent, H.nent);
    up(P->ndst, H.ndst);
    up(P->uent_off, H.uent_off);
    up(P->uent, H.uent);
    up(P->udst, H.udst);
    P->part.alloc(std::max<int64_t>(H.n_part, 1));
    P->txyz.alloc(H.n_tile_nodes + 1);
    k_tile_xyz<<<grid_for(H.n_tile_nodes, 256), 256, 0, s>>>(H.n_tile_nodes, P->tnode.get(), m->nodes4.get(),
                                                            P->txyz.get());
    UP3D_CHECK_LAUNCH();
    P->disp.alloc(12 * E);
    k_tile_disp<<<grid_for(12 * E, 256), 256, 0, s>>>(E, P->perm.get(), m->disp.get(), P->disp.get());
    UP3D_CHECK_LAUNCH();
    up(P->cn_off, H.cn_off);
    up(P->cn_idx, H.cn_idx);
    up(P->cn_dst, H.cn_dst);
    up(P->ce_off, H.ce_off);
    up(P->ce_idx, H.ce_idx);
    up(P->ce_dst, H.ce_dst);
    UP3D_CUDA(cudaStreamSynchronize(s));
    P->build_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    m->tiles = P;
}

}  // namespace up3d

using namespace up3d;

extern "C" {

int up3d_mesh_tile_info(up3d_mesh* m, int32_t tile_elems, up3d_tile_info* info, up3d_stream stream) {
    return guarded([&] {
        UP3D_REQUIRE(m && info, UP3D_ERR_ARGUMENT, "up3d_mesh_tile_info: null argument");
        ensure_tiles(m, tile_elems, m->tune.tile_stretch, S(stream));
        const TilePlan& P = *m->tiles;
        info->tile_elems = P.T;
        info->max_nodes = P.max_nodes;
        info->max_edges = P.max_edges;
        info->tile_stretch = P.stretch;
        info->n_tiles = P.n_tiles;
        info->n_tile_nodes = P.n_tile_nodes;
        info->n_tile_edges = P.n_tile_edges;
        info->n_partials = P.n_part;
        info->n_combined_nodes = P.n_cnode;
        info->n_combined_slots = P.n_cedge;
        info->build_s = P.build_s;
    });
}

// Host-side plan for tests and inspection (no device involved).
struct up3d_tile_plan {
    up3d::PlanHost H;
};

int up3d_tile_plan_host_create(const int32_t* elements, const int32_t* face_neighbors, const double* centroids,
                               int64_t n_nodes, int64_t n_tets, const int32_t* indptr, const int32_t* indices,
                               int32_t tile_elems, int32_t tile_stretch, up3d_tile_plan** out) {
    return guarded([&] {
        UP3D_REQUIRE(elements && face_neighbors && centroids && indptr && indices && out, UP3D_ERR_ARGUMENT,
                     "up3d_tile_plan_host_create: null argument");
        UP3D_REQUIRE(n_nodes > 0 && n_tets > 0 && n_tets < (1ll << 29), UP3D_ERR_VALUE,
                     "up3d_tile_plan_host_create: bad sizes");
        std::vector<int4> conn(n_tets), fn(n_tets);
        std::vector<double4> cen(n_tets);
        for (int64_t e = 0; e < n_tets; ++e) {
            const int32_t* c = elements + 4 * e;
            const int32_t* f = face_neighbors + 4 * e;
            for (int k = 0; k < 4; ++k)
                UP3D_REQUIRE(c[k] >= 0 && c[k] < n_nodes, UP3D_ERR_VALUE,
                             "up3d_tile_plan_host_create: node index out of range");
            conn[e] = make_int4(c[0], c[1], c[2], c[3]);
            fn[e] = make_int4(f[0], f[1], f[2], f[3]);
            cen[e] = make_double4(centroids[3 * e], centroids[3 * e + 1], centroids[3 * e + 2], 0.0);
        }
        const int64_t Z = indptr[n_nodes];
        std::vector<int32_t> ip(indptr, indptr + n_nodes + 1), ix(indices, indices + Z);
        auto* h = new up3d_tile_plan();
        try {
            h->H = build_plan_host(conn, fn, cen, n_nodes, ip, ix, tile_elems, tile_stretch);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int up3d_tile_plan_host_array(const up3d_tile_plan* h, const char* name, void* dst, int64_t* nbytes) {
    return guarded([&] {
        UP3D_REQUIRE(h && name && nbytes, UP3D_ERR_ARGUMENT, "up3d_tile_plan_host_array: null argument");
        const PlanHost& H = h->H;
        const std::string n(name);
        const void* src = nullptr;
        size_t bytes = 0;
        auto pick = [&](const auto& v) {
            src = v.data();
            bytes = sizeof(v[0]) * v.size();
        };
        if (n == "perm") pick(H.perm);
        else if (n == "iperm") pick(H.iperm);
        else if (n == "eoff") pick(H.eoff);
        else if (n == "noff") pick(H.noff);
        else if (n == "uoff") pick(H.uoff);
        else if (n == "tnode") pick(H.tnode);
        else if (n == "lconn") pick(H.lconn);
        else if (n == "nent_off") pick(H.nent_off);
        else if (n == "nent") pick(H.nent);
        else if (n == "ndst") pick(H.ndst);
        else if (n == "uent_off") pick(H.uent_off);
        else if (n == "uent") pick(H.uent);
        else if (n == "udst") pick(H.udst);
        else if (n == "cn_off") pick(H.cn_off);
        else if (n == "cn_idx") pick(H.cn_idx);
        else if (n == "cn_dst") pick(H.cn_dst);
        else if (n == "ce_off") pick(H.ce_off);
        else if (n == "ce_idx") pick(H.ce_idx);
        else if (n == "ce_dst") pick(H.ce_dst);
        else if (n == "fnbr") pick(H.fn_t);
        else UP3D_REQUIRE(false, UP3D_ERR_VALUE, "up3d_tile_plan_host_array: unknown array " + n);
        *nbytes = (int64_t)bytes;
        if (dst && bytes) std::memcpy(dst, src, bytes);
    });
}

int up3d_tile_plan_host_info(const up3d_tile_plan* h, up3d_tile_info* info) {
    return guarded([&] {
        UP3D_REQUIRE(h && info, UP3D_ERR_ARGUMENT, "up3d_tile_plan_host_info: null argument");
        const PlanHost& H = h->H;
        info->tile_elems = H.T;
        info->max_nodes = H.max_nodes;
        info->max_edges = H.max_edges;
        info->tile_stretch = H.stretch;
        info->n_tiles = H.n_tiles;
        info->n_tile_nodes = H.n_tile_nodes;
        info->n_tile_edges = H.n_tile_edges;
        info->n_partials = H.n_part;
        info->n_combined_nodes = (int64_t)H.cn_dst.size();
        info->n_combined_slots = (int64_t)H.ce_dst.size();
        info->build_s = 0.0;
    });
}

int up3d_tile_plan_host_destroy(up3d_tile_plan* h) {
    return guarded([&] { delete h; });
}

}  // extern "C"
