// Greedy facet patches (see patches.hpp).
#include "patches.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <utility>
#include <vector>

namespace litho_b200 {

namespace {

uint64_t spread3(uint32_t v) {  // 21 bits -> every third bit
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffull;
    x = (x | x << 16) & 0x1f0000ff0000ffull;
    x = (x | x << 8) & 0x100f00f00f00f00full;
    x = (x | x << 4) & 0x10c30c30c30c30c3ull;
    x = (x | x << 2) & 0x1249249249249249ull;
    return x;
}

}  // namespace

PatchTopology build_patches(int nv, const double* xyz, int nt, const int32_t* tri, int G, const int32_t* grpTriOff) {
    PatchTopology pt;
    pt.grpPatchOff.assign(1, 0);
    pt.facetOff.assign(1, 0);
    pt.vertOff.assign(1, 0);
    pt.edgeOff.assign(1, 0);
    pt.blobOff.assign(1, 0);
    // vertex -> facets incidence (all groups; filtered by group below)
    std::vector<int32_t> vfOff(nv + 1, 0), vf(3 * (size_t)nt);
    for (int k = 0; k < 3 * nt; ++k) vfOff[tri[k] + 1]++;
    for (int v = 0; v < nv; ++v) vfOff[v + 1] += vfOff[v];
    {
        std::vector<int32_t> fill(vfOff.begin(), vfOff.end() - 1);
        for (int k = 0; k < 3 * nt; ++k) vf[fill[tri[k]]++] = k / 3;
    }
    std::vector<uint8_t> assigned(nt, 0), queued(nt, 0);
    std::vector<int32_t> localOf(nv, -1);  // global vertex -> local index in the patch being grown
    std::vector<int32_t> cand;
    for (int g = 0; g < G; ++g) {
        const int f0 = grpTriOff[g], f1 = grpTriOff[g + 1];
        // seed order: Morton code of the facet centroids over the group's box
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        std::vector<double> cen(3 * (size_t)(f1 - f0));
        for (int f = f0; f < f1; ++f)
            for (int a = 0; a < 3; ++a) {
                const double c =
                    (xyz[3 * tri[3 * f] + a] + xyz[3 * tri[3 * f + 1] + a] + xyz[3 * tri[3 * f + 2] + a]) / 3.0;
                cen[3 * (f - f0) + a] = c;
                lo[a] = std::min(lo[a], c);
                hi[a] = std::max(hi[a], c);
            }
        const double span = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-30});
        std::vector<std::pair<uint64_t, int32_t>> order(f1 - f0);
        for (int f = f0; f < f1; ++f) {
            uint64_t key = 0;
            for (int a = 0; a < 3; ++a) {
                const double q = (cen[3 * (f - f0) + a] - lo[a]) / span * 2097151.0;
                key |= spread3(static_cast<uint32_t>(std::min(std::max(q, 0.0), 2097151.0))) << a;
            }
            order[f - f0] = {key, f};
        }
        std::sort(order.begin(), order.end());
        std::vector<int32_t> rank(f1 - f0);
        for (int i = 0; i < f1 - f0; ++i) rank[order[i].second - f0] = i;

        for (int oi = 0; oi < f1 - f0; ++oi) {
            const int seed = order[oi].second;
            if (assigned[seed]) continue;
            std::vector<int32_t> pf, pv;
            cand.clear();
            auto addFacet = [&](int f) {
                assigned[f] = 1;
                pf.push_back(f);
                for (int k = 0; k < 3; ++k) {
                    const int v = tri[3 * f + k];
                    if (localOf[v] >= 0) continue;
                    localOf[v] = static_cast<int32_t>(pv.size());
                    pv.push_back(v);
                    for (int j = vfOff[v]; j < vfOff[v + 1]; ++j) {
                        const int h = vf[j];
                        if (h >= f0 && h < f1 && !assigned[h] && !queued[h]) {
                            queued[h] = 1;
                            cand.push_back(h);
                        }
                    }
                }
            };
            addFacet(seed);
            while ((int)pf.size() < kPatchFacets) {
                int best = -1, bestNew = 4, bestRank = 0, bestPos = -1;
                for (int ci = 0; ci < (int)cand.size(); ++ci) {
                    const int h = cand[ci];
                    if (assigned[h]) continue;
                    int nnew = 0;
                    for (int k = 0; k < 3; ++k) nnew += localOf[tri[3 * h + k]] < 0;
                    if ((int)pv.size() + nnew > kPatchVerts) continue;
                    const int r = rank[h - f0];
                    if (nnew < bestNew || (nnew == bestNew && r < bestRank)) {
                        best = h;
                        bestNew = nnew;
                        bestRank = r;
                        bestPos = ci;
                    }
                }
                if (best < 0) break;
                cand[bestPos] = cand.back();
                cand.pop_back();
                addFacet(best);
            }
            for (int h : cand) queued[h] = 0;
            // edges: distinct unordered vertex pairs, at most two users each
            std::vector<uint32_t> einfo;
            std::vector<uint8_t> eslot;
            std::vector<uint32_t> corners;
            for (int lf = 0; lf < (int)pf.size(); ++lf) {
                const int f = pf[lf];
                uint32_t l[3];
                for (int k = 0; k < 3; ++k) l[k] = static_cast<uint32_t>(localOf[tri[3 * f + k]]);
                corners.push_back(l[0] | l[1] << 8 | l[2] << 16);
                for (int i = 0; i < 3; ++i) {
                    const uint32_t a = std::min(l[i], l[(i + 1) % 3]), b = std::max(l[i], l[(i + 1) % 3]);
                    int found = -1;
                    for (int e = 0; e < (int)einfo.size(); ++e)
                        if ((einfo[e] & 0xffffu) == (a | b << 8) && (einfo[e] >> 24) == (uint32_t)kNoFacet) {
                            found = e;
                            break;
                        }
                    if (found >= 0) {
                        einfo[found] = (einfo[found] & 0x00ffffffu) | (uint32_t)lf << 24;
                        eslot[found] = static_cast<uint8_t>(eslot[found] | i << 2);
                    } else {
                        einfo.push_back(a | b << 8 | (uint32_t)lf << 16 | (uint32_t)kNoFacet << 24);
                        eslot.push_back(static_cast<uint8_t>(i));
                    }
                }
            }
            for (int v : pv) localOf[v] = -1;
            pt.facets.insert(pt.facets.end(), pf.begin(), pf.end());
            pt.facetCorners.insert(pt.facetCorners.end(), corners.begin(), corners.end());
            pt.verts.insert(pt.verts.end(), pv.begin(), pv.end());
            pt.edgeInfo.insert(pt.edgeInfo.end(), einfo.begin(), einfo.end());
            pt.edgeSlot.insert(pt.edgeSlot.end(), eslot.begin(), eslot.end());
            pt.facetOff.push_back(static_cast<int32_t>(pt.facets.size()));
            pt.vertOff.push_back(static_cast<int32_t>(pt.verts.size()));
            pt.edgeOff.push_back(static_cast<int32_t>(pt.edgeInfo.size()));
            const int bytes = kPatchHeadBytes + (int)pv.size() * kPatchVertBytes +
                              (int)einfo.size() * kPatchEdgeBytes + (int)pf.size() * kPatchFacetBytes;
            pt.blobOff.push_back(pt.blobOff.back() + bytes);
            pt.P++;
        }
        pt.grpPatchOff.push_back(pt.P);
    }
    return pt;
}

}  // namespace litho_b200
