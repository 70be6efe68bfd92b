// Host-side validation, colouring and partition plan (see plan.h).
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

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

void rcb(int* ids, int n, int parts, int base, const float* xy, std::vector<int>& part_of) {
    if (parts <= 1 || n <= 1) {
        for (int i = 0; i < n; i++) part_of[ids[i]] = base;
        return;
    }
    float lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 2; d++) {
            lo[d] = std::min(lo[d], xy[2 * ids[i] + d]);
            hi[d] = std::max(hi[d], xy[2 * ids[i] + d]);
        }
    const int ax = (hi[0] - lo[0] >= hi[1] - lo[1]) ? 0 : 1;
    const int p1 = parts / 2;
    const int n1 = (int)((long long)n * p1 / parts);
    std::nth_element(ids, ids + n1, ids + n, [&](int a, int b) {
        float va = xy[2 * a + ax], vb = xy[2 * b + ax];
        return va < vb || (va == vb && a < b);
    });
    rcb(ids, n1, p1, base, xy, part_of);
    rcb(ids + n1, n - n1, parts - p1, base + p1, xy, part_of);
}

}  // namespace

std::string build_partition(const pg_problem& p, int G, HostPlan& plan) {
    const int Nn = plan.Nn, npe = plan.npe, C = plan.colors;
    if (G < 1) G = 1;
    if (G > std::max(Nn, 1)) G = std::max(Nn, 1);
    plan.G = G;
    std::vector<int> part_of(Nn, 0), ids(Nn);
    std::iota(ids.begin(), ids.end(), 0);
    rcb(ids.data(), Nn, G, 0, p.nodes, part_of);

    std::vector<int> elem_color(plan.Ne, 0);
    for (int c = 0; c < C; c++)
        for (uint32_t q = plan.color_offsets[c]; q < plan.color_offsets[c + 1]; q++)
            elem_color[plan.elements_by_color[q]] = c;

    std::vector<std::vector<int>> owned(G);
    for (int n = 0; n < Nn; n++) owned[part_of[n]].push_back(n);

    plan.node_off.assign(G + 1, 0);
    plan.nown.assign(G, 0);
    plan.elem_off.assign(G + 1, 0);
    plan.color_off.assign((size_t)G * (C + 1), 0);
    plan.nodes.clear();
    plan.elems.clear();
    plan.lnode.clear();
    plan.max_nloc = plan.max_nown = plan.max_nel = 0;

    std::vector<int> estamp(plan.Ne, -1), local(Nn, -1);
    std::vector<int> pel, ghosts;
    for (int g = 0; g < G; g++) {
        const std::vector<int>& own = owned[g];
        pel.clear();
        for (int n : own)
            for (int q = plan.inc_ptr[n]; q < plan.inc_ptr[n + 1]; q++) {
                int e = plan.inc_idx[q] / 4;
                if (estamp[e] != g) { estamp[e] = g; pel.push_back(e); }
            }
        std::sort(pel.begin(), pel.end(), [&](int a, int b) {
            return elem_color[a] < elem_color[b] || (elem_color[a] == elem_color[b] && a < b);
        });
        for (size_t i = 0; i < own.size(); i++) local[own[i]] = (int)i;
        ghosts.clear();
        for (int e : pel)
            for (int k = 0; k < npe; k++) {
                int n = (int)p.elements[(size_t)e * npe + k];
                if (part_of[n] != g && local[n] < 0) { local[n] = -2; ghosts.push_back(n); }
            }
        std::sort(ghosts.begin(), ghosts.end());
        for (size_t i = 0; i < ghosts.size(); i++) local[ghosts[i]] = (int)(own.size() + i);

        plan.nown[g] = (int)own.size();
        plan.nodes.insert(plan.nodes.end(), own.begin(), own.end());
        plan.nodes.insert(plan.nodes.end(), ghosts.begin(), ghosts.end());
        plan.node_off[g + 1] = (int)plan.nodes.size();
        const int ebase = (int)plan.elems.size();
        for (int c = 0; c <= C; c++) {
            // absolute offset of the first element of colour c within this part
            int cnt = 0;
            for (int e : pel)
                if (elem_color[e] < c) cnt++;
            plan.color_off[(size_t)g * (C + 1) + c] = ebase + cnt;
        }
        for (int e : pel) {
            plan.elems.push_back(e);
            for (int k = 0; k < npe; k++) plan.lnode.push_back(local[p.elements[(size_t)e * npe + k]]);
        }
        plan.elem_off[g + 1] = (int)plan.elems.size();
        plan.max_nloc = std::max(plan.max_nloc, (int)(own.size() + ghosts.size()));
        plan.max_nown = std::max(plan.max_nown, (int)own.size());
        plan.max_nel = std::max(plan.max_nel, (int)pel.size());
        for (int n : own) local[n] = -1;
        for (int n : ghosts) local[n] = -1;
    }
    return "";
}

uint64_t problem_hash(const pg_problem& p) {
    uint64_t h = 0x9e3779b97f4a7c15ull;
    auto mix = [&](uint64_t v) {
        h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
        h *= 0xff51afd7ed558ccdull;
        h ^= h >> 33;
    };
    auto bytes = [&](const void* d, size_t n) {
        if (!d) { mix(0xdeadull); return; }
        const unsigned char* b = (const unsigned char*)d;
        size_t i = 0;
        for (; i + 8 <= n; i += 8) {
            uint64_t v;
            std::memcpy(&v, b + i, 8);
            mix(v);
        }
        uint64_t tail = 0;
        std::memcpy(&tail, b + i, n - i);
        mix(tail ^ (uint64_t)n);
    };
    mix(p.node_count);
    mix(p.element_count);
    mix(p.nodes_per_element);
    mix(p.color_count);
    bytes(p.nodes, 2 * sizeof(float) * p.node_count);
    bytes(p.elements, sizeof(uint32_t) * p.nodes_per_element * p.element_count);
    if (p.color_count) {
        bytes(p.color_offsets, sizeof(uint32_t) * (p.color_count + 1));
        bytes(p.elements_by_color, sizeof(uint32_t) * p.element_count);
    }
    bytes(p.constrained, 3 * (size_t)p.node_count);
    double mat[3] = {p.E, p.nu, p.t};
    bytes(mat, sizeof(mat));
    bytes(p.elem_t, p.elem_t ? sizeof(float) * p.element_count : 0);
    return h;
}

}  // namespace pg
