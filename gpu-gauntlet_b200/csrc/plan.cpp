// Host-side validation, colouring and partition plan (see plan.h).
#include "plan.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <thread>

namespace pg {

namespace {

bool finite_f(const float* a, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!std::isfinite(a[i])) return false;
    return true;
}

}  // namespace

std::string validate_problem(const pg_problem& p, bool need_rhs) {
    if (p.nodes_per_element != 3 && p.nodes_per_element != 4)
        return "nodes_per_element must be 3 (DKT) or 4 (Q4)";
    if (p.node_count > (1u << 26) || p.element_count > (1u << 26))
        return "problem too large (node_count and element_count must be < 2^26)";
    if (p.node_count > 0 && !p.nodes) return "nodes is NULL";
    if (p.element_count > 0 && !p.elements) return "elements is NULL";
    if (p.node_count > 0 && !p.constrained) return "constrained is NULL";
    if (need_rhs && p.node_count > 0 && !p.F) return "F is NULL";
    if (!std::isfinite(p.E) || !std::isfinite(p.nu) || !std::isfinite(p.t))
        return "material E, nu, t must be finite";
    if (p.node_count && !finite_f(p.nodes, 2 * (size_t)p.node_count))
        return "node coordinates must be finite";
    if (p.elem_t && p.element_count && !finite_f(p.elem_t, p.element_count))
        return "elem_t must be finite";
    const size_t ne = (size_t)p.element_count * p.nodes_per_element;
    for (size_t i = 0; i < ne; i++)
        if (p.elements[i] >= p.node_count) return "element node index out of range";
    if (p.color_count > 0) {
        if (!p.color_offsets || !p.elements_by_color) return "colouring arrays are NULL";
        if (p.color_offsets[0] != 0 || p.color_offsets[p.color_count] != p.element_count)
            return "color_offsets must start at 0 and end at element_count";
        for (uint32_t c = 0; c < p.color_count; c++)
            if (p.color_offsets[c + 1] < p.color_offsets[c]) return "color_offsets must not decrease";
        std::vector<uint8_t> seen(p.element_count, 0);
        for (uint32_t i = 0; i < p.element_count; i++) {
            uint32_t e = p.elements_by_color[i];
            if (e >= p.element_count || seen[e]) return "elements_by_color must list every element once";
            seen[e] = 1;
        }
    }
    return "";
}

std::string build_structure(const pg_problem& p, HostPlan& plan) {
    const int Nn = (int)p.node_count, Ne = (int)p.element_count, npe = (int)p.nodes_per_element;
    plan.Nn = Nn;
    plan.Ne = Ne;
    plan.npe = npe;
    // node -> incident (element, position), element ids ascending
    plan.inc_ptr.assign(Nn + 1, 0);
    for (int e = 0; e < Ne; e++)
        for (int k = 0; k < npe; k++) plan.inc_ptr[p.elements[(size_t)e * npe + k] + 1]++;
    for (int n = 0; n < Nn; n++) plan.inc_ptr[n + 1] += plan.inc_ptr[n];
    plan.inc_idx.assign(plan.inc_ptr[Nn], 0);
    {
        std::vector<int> fill(plan.inc_ptr.begin(), plan.inc_ptr.end() - 1);
        for (int e = 0; e < Ne; e++)
            for (int k = 0; k < npe; k++)
                plan.inc_idx[fill[p.elements[(size_t)e * npe + k]]++] = e * 4 + k;
    }
    // colour of every element from the caller's lists
    std::vector<int> color(Ne, -1);
    bool valid = p.color_count > 0;
    if (valid) {
        for (uint32_t c = 0; c < p.color_count; c++)
            for (uint32_t q = p.color_offsets[c]; q < p.color_offsets[c + 1]; q++)
                color[p.elements_by_color[q]] = (int)c;
        // conflict check (verifyColoring, coloring.ts:188-225)
        std::vector<int> stamp(std::max<int>(p.color_count, 1), -1);
        for (int n = 0; n < Nn && valid; n++) {
            for (int q = plan.inc_ptr[n]; q < plan.inc_ptr[n + 1]; q++) {
                int c = color[plan.inc_idx[q] / 4];
                if (stamp[c] == n) { valid = false; break; }
                stamp[c] = n;
            }
        }
    }
    if (!valid && Ne > 0) {
        // greedy first-fit colouring in element order (coloring.ts:92-177)
        plan.recolored = p.color_count > 0;
        std::fill(color.begin(), color.end(), -1);
        std::vector<int> used(64, -1);
        for (int e = 0; e < Ne; e++) {
            for (int k = 0; k < npe; k++) {
                int n = (int)p.elements[(size_t)e * npe + k];
                for (int q = plan.inc_ptr[n]; q < plan.inc_ptr[n + 1]; q++) {
                    int nb = plan.inc_idx[q] / 4;
                    if (nb != e && color[nb] >= 0) {
                        if (color[nb] >= (int)used.size()) used.resize(color[nb] * 2 + 2, -1);
                        used[color[nb]] = e;
                    }
                }
            }
            int c = 0;
            while (c < (int)used.size() && used[c] == e) c++;
            color[e] = c;
        }
    }
    int C = 1;
    for (int e = 0; e < Ne; e++) C = std::max(C, color[e] + 1);
    plan.colors = C;
    plan.color_offsets.assign(C + 1, 0);
    for (int e = 0; e < Ne; e++) plan.color_offsets[color[e] + 1]++;
    for (int c = 0; c < C; c++) plan.color_offsets[c + 1] += plan.color_offsets[c];
    plan.elements_by_color.assign(Ne, 0);
    {
        std::vector<uint32_t> fill(plan.color_offsets.begin(), plan.color_offsets.end() - 1);
        if (valid) {
            for (uint32_t c = 0; c < p.color_count; c++)
                for (uint32_t q = p.color_offsets[c]; q < p.color_offsets[c + 1]; q++)
                    plan.elements_by_color[fill[c]++] = p.elements_by_color[q];
        } else {
            for (int e = 0; e < Ne; e++) plan.elements_by_color[fill[color[e]]++] = (uint32_t)e;
        }
    }
    return "";
}

namespace {

// Order-preserving map of a finite float to an unsigned key (-0 as +0, so
// keys compare as the values do).
inline uint32_t float_key(float v) {
    if (v == 0.0f) v = 0.0f;
    uint32_t u;
    std::memcpy(&u, &v, sizeof u);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct SortKey {
    uint64_t k;  // primary coordinate key << 32 | secondary coordinate key
    int id;
};

// Stable sort of v[b, e) by k: equal keys keep their incoming order.
// Meshes numbered row by row arrive sorted by (y, x) already.
void sort_keys(std::vector<SortKey>& v, size_t b, size_t e) {
    auto less = [](const SortKey& u, const SortKey& w) { return u.k < w.k; };
    if (!std::is_sorted(v.begin() + b, v.begin() + e, less)) std::stable_sort(v.begin() + b, v.begin() + e, less);
}

}  // namespace

// Near-square partition of a node cloud into G parts (see plan.h).
void strip_partition(const float* xy, int Nn, int G, std::vector<int>& part_of) {
    part_of.assign(Nn, 0);
    if (G <= 1 || Nn == 0) return;
    float lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (int n = 0; n < Nn; n++)
        for (int d = 0; d < 2; d++) {
            lo[d] = std::min(lo[d], xy[2 * n + d]);
            hi[d] = std::max(hi[d], xy[2 * n + d]);
        }
    const double W = std::max(1e-30, (double)hi[0] - lo[0]), H = std::max(1e-30, (double)hi[1] - lo[1]);
    int R = (int)std::lround(std::sqrt((double)G * H / W));
    R = std::max(1, std::min(R, G));
    // first by (y, x, id), then each strip by (x, y, id): stable sorts of the
    // packed coordinate keys, the ids entering in increasing order (and a
    // strip's equal (x, y) pairs keep the id order of the first sort)
    std::vector<SortKey> keys(Nn);
    std::vector<uint32_t> kx(Nn), ky(Nn);
    for (int n = 0; n < Nn; n++) {
        kx[n] = float_key(xy[2 * n]);
        ky[n] = float_key(xy[2 * n + 1]);
        keys[n] = SortKey{(uint64_t)ky[n] << 32 | kx[n], n};
    }
    sort_keys(keys, 0, (size_t)Nn);
    int part = 0;
    long long done_blocks = 0;
    int start = 0;
    for (int s = 0; s < R; s++) {
        const int blocks = G / R + (s < G % R ? 1 : 0);
        done_blocks += blocks;
        const int end = (int)((long long)Nn * done_blocks / G);
        for (int i = start; i < end; i++) {
            const int n = keys[i].id;
            keys[i].k = (uint64_t)kx[n] << 32 | ky[n];
        }
        sort_keys(keys, (size_t)start, (size_t)end);
        const int len = end - start;
        for (int b = 0; b < blocks; b++) {
            const int b0 = start + (int)((long long)len * b / blocks);
            const int b1 = start + (int)((long long)len * (b + 1) / blocks);
            for (int i = b0; i < b1; i++) part_of[keys[i].id] = part;
            part++;
        }
        start = end;
    }
}

std::string build_partition(const pg_problem& p, int G, int rings, HostPlan& plan) {
    const int Nn = plan.Nn, npe = plan.npe;
    if (G < 1) G = 1;
    if (G > std::max(Nn, 1)) G = std::max(Nn, 1);
    plan.G = G;
    plan.rings = rings == 2 ? 2 : 1;
    std::vector<int> part_of;
    strip_partition(p.nodes, Nn, G, part_of);

    std::vector<std::vector<int>> owned(G);
    for (int n = 0; n < Nn; n++) owned[part_of[n]].push_back(n);

    plan.node_off.assign(G + 1, 0);
    plan.nown.assign(G, 0);
    plan.task_off.assign(G + 1, 0);
    plan.tp_off.assign(G + 1, 0);
    plan.nodes.clear();
    plan.task_elem.clear();
    plan.task_pos.clear();
    plan.task_nodes.clear();
    plan.tptr.clear();
    plan.n1.assign(G, 0);
    plan.max_nloc = plan.max_nown = plan.max_ntask = plan.max_ntask_own = plan.max_n1 = 0;

    // Each part's lists are built independently (host threads over parts,
    // each with its own node -> local-index map), then concatenated in part
    // order.
    struct PartOut {
        std::vector<int> nodes, tptr, task_elem;
        std::vector<uint8_t> task_pos;
        std::vector<uint16_t> task_nodes;
        int nown = 0, n1 = 0, nloc = 0, ntask_own = 0;
        bool too_large = false;
    };
    std::vector<PartOut> out(G);
    const bool two = rings == 2;
    auto build_part = [&](int g, std::vector<int>& local, std::vector<int>& ghosts, std::vector<int>& ring2) {
        // fills `dst` (sorted) with the nodes of elements around `from` not yet numbered
        auto next_ring = [&](const std::vector<int>& from, std::vector<int>& dst) {
            dst.clear();
            for (int n : from)
                for (int q = plan.inc_ptr[n]; q < plan.inc_ptr[n + 1]; q++) {
                    const int e = plan.inc_idx[q] / 4;
                    for (int k = 0; k < npe; k++) {
                        const int m = (int)p.elements[(size_t)e * npe + k];
                        if (local[m] == -1) { local[m] = -2; dst.push_back(m); }
                    }
                }
            std::sort(dst.begin(), dst.end());
        };
        PartOut& o = out[g];
        const std::vector<int>& own = owned[g];
        for (size_t i = 0; i < own.size(); i++) local[own[i]] = (int)i;
        next_ring(own, ghosts);
        for (size_t i = 0; i < ghosts.size(); i++) local[ghosts[i]] = (int)(own.size() + i);
        ring2.clear();
        if (two) {
            next_ring(ghosts, ring2);
            for (size_t i = 0; i < ring2.size(); i++) local[ring2[i]] = (int)(own.size() + ghosts.size() + i);
        }
        o.nloc = (int)(own.size() + ghosts.size() + ring2.size());
        o.nown = (int)own.size();
        o.n1 = two ? (int)(own.size() + ghosts.size()) : (int)own.size();
        o.too_large = o.nloc > 65535;
        if (!o.too_large) {
            o.nodes.reserve(o.nloc);
            o.nodes.insert(o.nodes.end(), own.begin(), own.end());
            o.nodes.insert(o.nodes.end(), ghosts.begin(), ghosts.end());
            o.nodes.insert(o.nodes.end(), ring2.begin(), ring2.end());
            const int ntn = o.n1;
            size_t ntask = 0;
            for (int i = 0; i < ntn; i++) {
                const int n = i < (int)own.size() ? own[i] : ghosts[i - own.size()];
                ntask += (size_t)(plan.inc_ptr[n + 1] - plan.inc_ptr[n]);
            }
            o.tptr.resize(ntn + 1);
            o.task_elem.resize(ntask);
            o.task_pos.resize(ntask);
            o.task_nodes.resize(ntask * npe);
            int* te = o.task_elem.data();
            uint8_t* tpos = o.task_pos.data();
            uint16_t* tnod = o.task_nodes.data();
            int t = 0;
            for (int i = 0; i < ntn; i++) {
                const int n = i < (int)own.size() ? own[i] : ghosts[i - own.size()];
                if (i == (int)own.size()) o.ntask_own = t;
                o.tptr[i] = t;
                for (int q = plan.inc_ptr[n]; q < plan.inc_ptr[n + 1]; q++, t++) {
                    const int e = plan.inc_idx[q] / 4, k = plan.inc_idx[q] % 4;
                    te[t] = e;
                    tpos[t] = (uint8_t)k;
                    const uint32_t* en = p.elements + (size_t)e * npe;
                    uint16_t* dst = tnod + (size_t)t * npe;
                    for (int j = 0, kj = k; j < npe; j++, kj = kj + 1 == npe ? 0 : kj + 1)
                        dst[j] = (uint16_t)local[en[kj]];
                }
            }
            if (ntn == (int)own.size()) o.ntask_own = t;
            o.tptr[ntn] = t;
        }
        for (int n : own) local[n] = -1;
        for (int n : ghosts) local[n] = -1;
        for (int n : ring2) local[n] = -1;
    };
    const int nth = std::max(1, std::min({(int)std::thread::hardware_concurrency(), 16, G, 1 + Nn / 4096}));
    std::atomic<int> next{0};
    std::atomic<bool> failed{false};
    auto worker = [&]() {
        // an exception must not leave a worker thread (std::terminate):
        // recorded here, raised again on the calling thread
        try {
            std::vector<int> local(Nn, -1), ghosts, ring2;
            for (int g; !failed && (g = next.fetch_add(1)) < G;) build_part(g, local, ghosts, ring2);
        } catch (...) {
            failed = true;
        }
    };
    {
        std::vector<std::thread> th;
        for (int t = 1; t < nth; t++) th.emplace_back(worker);
        worker();
        for (auto& t : th) t.join();
    }
    if (failed) throw std::bad_alloc();
    size_t tot_nodes = 0, tot_tasks = 0, tot_tptr = 0;
    for (int g = 0; g < G; g++) {
        if (out[g].too_large) return "a part has more than 65535 local nodes: use more ctas";
        tot_nodes += out[g].nodes.size();
        tot_tasks += out[g].task_elem.size();
        tot_tptr += out[g].tptr.size();
    }
    plan.nodes.reserve(tot_nodes);
    plan.task_elem.reserve(tot_tasks);
    plan.task_pos.reserve(tot_tasks);
    plan.task_nodes.reserve(tot_tasks * npe);
    plan.tptr.reserve(tot_tptr);
    for (int g = 0; g < G; g++) {
        const PartOut& o = out[g];
        plan.nown[g] = o.nown;
        plan.n1[g] = o.n1;
        plan.nodes.insert(plan.nodes.end(), o.nodes.begin(), o.nodes.end());
        plan.node_off[g + 1] = (int)plan.nodes.size();
        plan.tp_off[g] = (int)plan.tptr.size();
        plan.tptr.insert(plan.tptr.end(), o.tptr.begin(), o.tptr.end());
        plan.task_elem.insert(plan.task_elem.end(), o.task_elem.begin(), o.task_elem.end());
        plan.task_pos.insert(plan.task_pos.end(), o.task_pos.begin(), o.task_pos.end());
        plan.task_nodes.insert(plan.task_nodes.end(), o.task_nodes.begin(), o.task_nodes.end());
        plan.task_off[g + 1] = (int)plan.task_elem.size();
        plan.max_nloc = std::max(plan.max_nloc, o.nloc);
        plan.max_nown = std::max(plan.max_nown, o.nown);
        plan.max_n1 = std::max(plan.max_n1, o.n1);
        plan.max_ntask = std::max(plan.max_ntask, (int)o.task_elem.size());
        plan.max_ntask_own = std::max(plan.max_ntask_own, o.ntask_own);
    }
    plan.tp_off[G] = (int)plan.tptr.size();
    return "";
}

// sum_{k in [k0, k1)} a[k] b[k] in four interleaved partial sums (the
// dependent additions of a single running sum would bound the dense steps
// of the coarse set-up by the adder's latency)
static double dot4(const double* a, const double* b, int k0, int k1) {
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {
        s0 += a[k] * b[k];
        s1 += a[k + 1] * b[k + 1];
        s2 += a[k + 2] * b[k + 2];
        s3 += a[k + 3] * b[k + 3];
    }
    for (; k < k1; k++) s0 += a[k] * b[k];
    return (s0 + s1) + (s2 + s3);
}

std::string build_coarse_meta(const pg_problem& p, HostPlan& plan) {
    const int G = plan.G, Nn = plan.Nn;
    const int C = 3 * G;
    plan.C = C;
    plan.coarse_owner.assign(Nn, 0);
    plan.coarse_geom.assign(3 * (size_t)G, 0.0);
    std::vector<int>& owner = plan.coarse_owner;
    for (int g = 0; g < G; g++) {
        const int n0 = plan.node_off[g], no = plan.nown[g];
        double sx = 0, sy = 0, lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
        for (int k = 0; k < no; k++) {
            const int n = plan.nodes[n0 + k];
            owner[n] = g;
            const double x = p.nodes[2 * n], y = p.nodes[2 * n + 1];
            sx += x;
            sy += y;
            lo[0] = std::min(lo[0], x); hi[0] = std::max(hi[0], x);
            lo[1] = std::min(lo[1], y); hi[1] = std::max(hi[1], y);
        }
        double cx = 0, cy = 0, ih = 1.0;
        if (no > 0) {
            cx = sx / no;
            cy = sy / no;
            const double h = std::max(hi[0] - lo[0], hi[1] - lo[1]);
            ih = h > 0 ? 1.0 / h : 1.0;
        }
        plan.coarse_geom[3 * g] = cx;
        plan.coarse_geom[3 * g + 1] = cy;
        plan.coarse_geom[3 * g + 2] = ih;
    }
    // per part: aggregates of its local nodes, node slots and basis data
    plan.node_basis.assign(3 * plan.nodes.size(), 0.0);
    plan.node_slot.assign(plan.nodes.size(), 0);
    plan.cagg_off.assign(G + 1, 0);
    plan.cagg.clear();
    plan.ainv_off.assign(G + 1, 0);
    plan.ainv_src.clear();
    plan.ainv.clear();
    plan.max_kagg = 0;
    std::vector<int> slot_of(G, -1);
    for (int g = 0; g < G; g++) {
        // aggregates of the nodes where the part forms u: owned and ring 1
        // (ring-2 nodes, rings = 2, carry only r, s and w: slot 0, unused)
        const int n0 = plan.node_off[g], nl = plan.node_off[g + 1] - n0;
        const int nu = plan.rings == 2 ? plan.n1[g] : nl;
        std::vector<int> list = {g};
        slot_of[g] = 0;
        for (int k = 0; k < nu; k++) {
            const int a = owner[plan.nodes[n0 + k]];
            if (slot_of[a] < 0) { slot_of[a] = (int)list.size(); list.push_back(a); }
        }
        for (int k = 0; k < nl; k++) {
            const int n = plan.nodes[n0 + k], a = owner[n];
            const double* ge = plan.coarse_geom.data() + 3 * a;
            plan.node_slot[n0 + k] = k < nu ? slot_of[a] : 0;
            plan.node_basis[3 * (n0 + k)] = (p.nodes[2 * n] - ge[0]) * ge[2];
            plan.node_basis[3 * (n0 + k) + 1] = (p.nodes[2 * n + 1] - ge[1]) * ge[2];
            plan.node_basis[3 * (n0 + k) + 2] = ge[2];
        }
        plan.ainv_off[g] = (int)plan.ainv_src.size();
        for (int a : list)
            for (int m = 0; m < 3; m++) plan.ainv_src.push_back(3 * a + m);
        plan.cagg.insert(plan.cagg.end(), list.begin(), list.end());
        plan.cagg_off[g + 1] = (int)plan.cagg.size();
        plan.max_kagg = std::max(plan.max_kagg, (int)list.size());
        for (int a : list) slot_of[a] = -1;
    }
    plan.ainv_off[G] = (int)plan.ainv_src.size();
    return "";
}

std::string build_coarse(const pg_problem& p, const std::vector<double>& ke64, HostPlan& plan) {
    std::string e = build_coarse_meta(p, plan);
    if (!e.empty()) return e;
    const int Nn = plan.Nn, npe = plan.npe, nd = 3 * npe;
    const int C = plan.C;
    const std::vector<int>& owner = plan.coarse_owner;
    const std::vector<double>& geom = plan.coarse_geom;
    (void)Nn;
    // basis of node n in mode m, DOF d (masked by constraints); Phi[d][m]
    auto phi = [&](int n, double Phi[3][3]) {
        const int a = owner[n];
        const double ih = geom[3 * a + 2];
        const double dx = (p.nodes[2 * n] - geom[3 * a]) * ih, dy = (p.nodes[2 * n + 1] - geom[3 * a + 1]) * ih;
        const double v[3][3] = {{1.0, dy, dx}, {0.0, ih, 0.0}, {0.0, 0.0, -ih}};
        for (int d = 0; d < 3; d++)
            for (int m = 0; m < 3; m++) Phi[d][m] = p.constrained[3 * n + d] ? 0.0 : v[d][m];
    };
    // A_c = P^T K P, element by element
    std::vector<double> Ac((size_t)C * C, 0.0);
    const size_t kk = (size_t)nd * nd;
    for (int e = 0; e < plan.Ne; e++) {
        const double* K = ke64.data() + (size_t)e * kk;
        double Ph[4][3][3];
        int ag[4];
        for (int i = 0; i < npe; i++) {
            const int n = (int)p.elements[(size_t)e * npe + i];
            phi(n, Ph[i]);
            ag[i] = owner[n];
        }
        for (int i = 0; i < npe; i++)
            for (int j = 0; j < npe; j++) {
                double T[3][3];  // K_ij Phi_j
                for (int d = 0; d < 3; d++)
                    for (int m = 0; m < 3; m++) {
                        double acc = 0;
                        for (int f = 0; f < 3; f++) acc += K[(3 * i + d) * nd + 3 * j + f] * Ph[j][f][m];
                        T[d][m] = acc;
                    }
                for (int mi = 0; mi < 3; mi++)
                    for (int mj = 0; mj < 3; mj++) {
                        double acc = 0;
                        for (int d = 0; d < 3; d++) acc += Ph[i][d][mi] * T[d][mj];
                        Ac[(size_t)(3 * ag[i] + mi) * C + 3 * ag[j] + mj] += acc;
                    }
            }
    }
    // Cholesky with dependent modes dropped, then the explicit inverse
    std::vector<double> Lm((size_t)C * C, 0.0);
    std::vector<char> keep(C, 1);
    double dmax = 0;
    for (int i = 0; i < C; i++) dmax = std::max(dmax, Ac[(size_t)i * C + i]);
    plan.dropped_modes = 0;
    for (int j = 0; j < C; j++) {
        const double* lrow = Lm.data() + (size_t)j * C;
        const double d = Ac[(size_t)j * C + j] - dot4(lrow, lrow, 0, j);
        if (!(d > 1e-13 * dmax)) {
            keep[j] = 0;
            plan.dropped_modes++;
            continue;
        }
        const double ljj = std::sqrt(d);
        Lm[(size_t)j * C + j] = ljj;
        for (int i = j + 1; i < C; i++) {
            const double s = Ac[(size_t)i * C + j] - dot4(Lm.data() + (size_t)i * C, lrow, 0, j);
            Lm[(size_t)i * C + j] = s / ljj;
        }
    }
    // inverse of L (lower), dropped columns stay zero; kept transposed
    // (Lt[j][k] = (L^-1)[k][j]) so that both loops below run along rows
    std::vector<double> Lt((size_t)C * C, 0.0);
    for (int j = 0; j < C; j++) {
        if (!keep[j]) continue;
        double* lj = Lt.data() + (size_t)j * C;
        lj[j] = 1.0 / Lm[(size_t)j * C + j];
        for (int i = j + 1; i < C; i++) {
            if (!keep[i]) continue;
            const double* li = Lm.data() + (size_t)i * C;
            lj[i] = -dot4(li, lj, j, i) / li[i];
        }
    }
    std::vector<double> Ainv((size_t)C * C, 0.0);  // L^-T L^-1
    for (int i = 0; i < C; i++)
        for (int j = 0; j <= i; j++) {
            const double s = dot4(Lt.data() + (size_t)i * C, Lt.data() + (size_t)j * C, i, C);
            Ainv[(size_t)i * C + j] = s;
            Ainv[(size_t)j * C + i] = s;
        }
    // each part's rows of A_c^-1 (3 per aggregate of its list)
    plan.ainv.resize(plan.ainv_src.size() * (size_t)C);
    for (size_t r = 0; r < plan.ainv_src.size(); r++)
        std::copy(Ainv.begin() + (size_t)plan.ainv_src[r] * C, Ainv.begin() + (size_t)(plan.ainv_src[r] + 1) * C,
                  plan.ainv.begin() + r * C);
    plan.coarse = true;
    return "";
}

std::string schedule_batch(const std::vector<int>& nodes, const std::vector<int>& caps,
                           const std::vector<int>& kinds, int sms, BatchSchedule& out, int part_nodes) {
    const double target = part_nodes > 0 ? part_nodes : 400.0;
    out = BatchSchedule{};
    const int count = (int)nodes.size();
    if (count == 0) return "empty batch";
    if (sms < 1 || (int)caps.size() != count || (int)kinds.size() != count) return "no blocks to schedule";
    int top = 1;  // largest power of two <= sms
    while (top * 2 <= sms) top *= 2;
    std::vector<int> d(count);
    std::vector<double> w(count);
    for (int i = 0; i < count; i++) {
        const double n = std::max(1, nodes[i]);
        const int cap = std::max(1, caps[i]);
        int need = 1;
        while (need < std::ceil(n / cap)) need *= 2;
        if (need > top) {
            if ((double)sms * cap < n) return "a plate of the batch needs more blocks than the device has";
            need = sms;
        }
        const int pref = std::max(1, (int)std::lround(std::exp2(std::round(std::log2(std::max(1.0, n / target))))));
        d[i] = std::max(need, std::min(top, pref));
        w[i] = std::sqrt(n) * (n + 300.0 * d[i]);
    }
    out.plate_phase.assign(count, -1);
    out.plate_team.assign(count, -1);
    out.plate_size = d;
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return w[a] > w[b]; });
    std::vector<int> ks;
    for (int i = 0; i < count; i++)
        if (std::find(ks.begin(), ks.end(), kinds[i]) == ks.end()) ks.push_back(kinds[i]);
    std::sort(ks.rbegin(), ks.rend());
    for (int kind : ks) {
    // team sizes of this kind, largest first, first-fit into phases (one team
    // of each size fits)
    std::vector<int> cs;
    for (int i = 0; i < count; i++)
        if (kinds[i] == kind && std::find(cs.begin(), cs.end(), d[i]) == cs.end()) cs.push_back(d[i]);
    std::sort(cs.rbegin(), cs.rend());
    std::vector<std::vector<int>> phase_sizes;
    std::vector<int> phase_sum;
    for (int c : cs) {
        size_t ph = 0;
        while (ph < phase_sizes.size() && phase_sum[ph] + c > sms) ph++;
        if (ph == phase_sizes.size()) {
            phase_sizes.emplace_back();
            phase_sum.push_back(0);
        }
        phase_sizes[ph].push_back(c);
        phase_sum[ph] += c;
    }
    for (size_t ph = 0; ph < phase_sizes.size(); ph++) {
        const std::vector<int>& pc = phase_sizes[ph];  // descending
        const int nc = (int)pc.size();
        std::vector<double> W(nc, 0.0);
        std::vector<int> teams(nc, 1), nplates(nc, 0);
        for (int i = 0; i < count; i++) {
            const auto it = std::find(pc.begin(), pc.end(), d[i]);
            if (kinds[i] != kind || it == pc.end()) continue;
            W[it - pc.begin()] += w[i];
            nplates[it - pc.begin()]++;
        }
        int used = phase_sum[ph];
        for (;;) {  // one more team to the size with the most work per block
            int best = -1;
            double bw = 0.0;
            for (int k = 0; k < nc; k++) {
                if (used + pc[k] > sms || teams[k] >= nplates[k]) continue;
                const double per = W[k] / ((double)teams[k] * pc[k]);
                if (per > bw) { bw = per; best = k; }
            }
            if (best < 0) break;
            teams[best]++;
            used += pc[best];
        }
        BatchPhase P;
        P.kind = kind;
        for (int k = 0; k < nc; k++)
            for (int t = 0; t < teams[k]; t++) {
                P.team_base.push_back(P.grid);
                P.team_size.push_back(pc[k]);
                P.grid += pc[k];
            }
        const int T = (int)P.team_size.size();
        P.team_load.assign(T, 0.0);
        std::vector<std::vector<int>> q(T);
        for (int i : order) {
            if (kinds[i] != kind || std::find(pc.begin(), pc.end(), d[i]) == pc.end()) continue;
            int bt = -1;
            for (int t = 0; t < T; t++)
                if (P.team_size[t] == d[i] && (bt < 0 || P.team_load[t] < P.team_load[bt])) bt = t;
            out.plate_phase[i] = (int)out.phases.size();
            out.plate_team[i] = bt;
            P.team_load[bt] += w[i];
            q[bt].push_back(i);
        }
        P.queue_off.assign(T + 1, 0);
        for (int t = 0; t < T; t++) {
            P.queue_off[t + 1] = P.queue_off[t] + (int)q[t].size();
            P.queue.insert(P.queue.end(), q[t].begin(), q[t].end());
        }
        // the dynamic queues: one per class (team size), largest work first
        std::vector<std::vector<int>> cq(nc);
        for (int i : order) {
            if (kinds[i] != kind) continue;
            const auto it = std::find(pc.begin(), pc.end(), d[i]);
            if (it != pc.end()) cq[it - pc.begin()].push_back(i);
        }
        P.class_off.assign(nc + 1, 0);
        for (int k = 0; k < nc; k++) {
            P.class_off[k + 1] = P.class_off[k] + (int)cq[k].size();
            P.class_queue.insert(P.class_queue.end(), cq[k].begin(), cq[k].end());
        }
        P.log_off.assign(T + 1, 0);
        for (int t = 0; t < T; t++) {
            const int k = (int)(std::find(pc.begin(), pc.end(), P.team_size[t]) - pc.begin());
            P.team_class.push_back(k);
            P.log_off[t + 1] = P.log_off[t] + (int)cq[k].size();
        }
        out.phases.push_back(std::move(P));
    }
    }
    return "";
}

}  // namespace pg
