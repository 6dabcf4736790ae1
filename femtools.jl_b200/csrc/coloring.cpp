// coloring.cpp — element colouring for conflict-free scatters (host code).
//
// color_mesh_greedy (src/mesh/coloring.jl:26-50): elements are visited in order
// and each takes the smallest positive colour not used by any element that shares
// a node with it, so elements of one colour share no node and a launch over one
// colour can scatter with plain adds. generate_element_groups (:77-81) lists the
// elements of each colour in ascending order.
#include <cstdint>
#include <vector>

#include "../../include/femtools_b200.h"

extern "C" {

int femb200_color_mesh(const int32_t* el2n, int32_t nv, int64_t nels, int64_t nnodes, int32_t* colors,
                       int32_t* ncolors) {
    if (!el2n || !colors || !ncolors || nv < 1 || nels < 0 || nnodes < 0) return FEMB200_EINVAL;
    // node → elements (generate_node2element, src/mesh/connectivity.jl:341), as CSR
    std::vector<int64_t> start(nnodes + 1, 0);
    for (int64_t e = 0; e < nels; ++e)
        for (int32_t i = 0; i < nv; ++i) {
            const int32_t n = el2n[(int64_t)nv * e + i];
            if (n < 1 || n > nnodes) return FEMB200_EINVAL;
            ++start[n];
        }
    for (int64_t n = 0; n < nnodes; ++n) start[n + 1] += start[n];
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    std::vector<int64_t> n2el(start[nnodes]);
    for (int64_t e = 0; e < nels; ++e)
        for (int32_t i = 0; i < nv; ++i) n2el[fill[el2n[(int64_t)nv * e + i] - 1]++] = e;
    // colours seen around the current element, stamped with its index
    std::vector<int64_t> stamp(1, -1);
    int32_t maxc = 0;
    for (int64_t e = 0; e < nels; ++e) colors[e] = 0;
    for (int64_t e = 0; e < nels; ++e) {
        for (int32_t i = 0; i < nv; ++i) {
            const int32_t n = el2n[(int64_t)nv * e + i] - 1;
            for (int64_t k = start[n]; k < start[n + 1]; ++k) {
                const int32_t c = colors[n2el[k]];
                if (c != 0) {
                    if ((size_t)c >= stamp.size()) stamp.resize((size_t)c + 1, -1);
                    stamp[c] = e;
                }
            }
        }
        int32_t c = 1;
        while ((size_t)c < stamp.size() && stamp[c] == e) ++c;
        colors[e] = c;
        if (c > maxc) maxc = c;
    }
    *ncolors = maxc;
    return FEMB200_OK;
}

int femb200_color_groups(const int32_t* colors, int64_t nels, int32_t ncolors, int64_t* offsets, int32_t* elements) {
    if (!colors || !offsets || !elements || nels < 0 || ncolors < 0) return FEMB200_EINVAL;
    for (int32_t c = 0; c <= ncolors; ++c) offsets[c] = 0;
    for (int64_t e = 0; e < nels; ++e) {
        if (colors[e] < 1 || colors[e] > ncolors) return FEMB200_EINVAL;
        ++offsets[colors[e]];
    }
    for (int32_t c = 0; c < ncolors; ++c) offsets[c + 1] += offsets[c];
    std::vector<int64_t> fill(offsets, offsets + ncolors);
    for (int64_t e = 0; e < nels; ++e) elements[fill[colors[e] - 1]++] = (int32_t)(e + 1);
    return FEMB200_OK;
}

}  // extern "C"
