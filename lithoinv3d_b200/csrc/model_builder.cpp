// Host-side lithology model bookkeeping (setup time).  See model_builder.hpp.
#include "model_builder.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <set>
#include <unordered_map>

namespace litho_b200 {

namespace {
inline double dist(const Vec3& a, const Vec3& b) {
    double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return std::sqrt(dx * dx + dy * dy + dz * dz);
}
inline int64_t quantize(double v) { return static_cast<int64_t>(std::round(v * 1e6)); }
struct PosKey {
    int64_t x, y, z;
    bool operator<(const PosKey& o) const {
        if (x != o.x) return x < o.x;
        if (y != o.y) return y < o.y;
        return z < o.z;
    }
};
}  // namespace

// SurfaceMesh::isPaddingVertex, surface_mesh.cpp:676-685.
bool Mesh::isPadding(uint32_t v) const {
    if (paddingRings <= 0) return false;
    int full = interiorGridDim + 2 * paddingRings;
    int r = static_cast<int>(v) / full, c = static_cast<int>(v) % full;
    return r < paddingRings || r >= paddingRings + interiorGridDim || c < paddingRings ||
           c >= paddingRings + interiorGridDim;
}

// SurfaceMesh::isControlPoint, surface_mesh.cpp:603-608: a vertex is a control
// point when CP mode is off, or when its weight row is exactly {(self, 1.0)}.
bool Mesh::isControlPoint(uint32_t v) const {
    if (cpStride <= 0) return true;
    if (cpWeights.empty()) return true;
    return cpWeights[v].size() == 1 && cpWeights[v][0].second == 1.0;
}

// SurfaceMesh::rebuildDofMappings, surface_mesh.cpp:91-172.
void Mesh::rebuildDofMappings() {
    dofs.clear();
    for (uint32_t v = 0; v < vertexCount(); ++v) {
        if (isPadding(v)) continue;
        if (cpStride > 0 && !isControlPoint(v)) continue;
        switch (freedom[v]) {
            case FIXED: break;
            case Z_ONLY: dofs.push_back({v, 2}); break;
            case X_ONLY: dofs.push_back({v, 0}); break;
            case Y_ONLY: dofs.push_back({v, 1}); break;
            case ALONG_VECTOR: dofs.push_back({v, 0}); break;
            case XY_FREE: dofs.push_back({v, 0}); dofs.push_back({v, 1}); break;
            case XZ_FREE: dofs.push_back({v, 0}); dofs.push_back({v, 2}); break;
            case YZ_FREE: dofs.push_back({v, 1}); dofs.push_back({v, 2}); break;
            case XYZ_FREE:
                dofs.push_back({v, 0}); dofs.push_back({v, 1}); dofs.push_back({v, 2});
                break;
            default: break;
        }
    }
}

// SurfaceMesh::setControlPointsExplicit, surface_mesh.cpp:544-601: explicit
// control points; every other vertex is inverse-distance weighted from its
// K = 4 nearest control points (ties broken by control-point index).
uint32_t Mesh::setControlPointsExplicit(const std::vector<uint32_t>& cps) {
    cpStride = 1;
    cpIndices = cps;
    cpWeights.clear();
    uint32_t nv = vertexCount(), nc = static_cast<uint32_t>(cpIndices.size());
    if (nc < 2 || nv < 2) {
        cpStride = 0;
        cpIndices.clear();
        return 0;
    }
    std::unordered_map<uint32_t, uint32_t> cpOf;
    for (uint32_t ci = 0; ci < nc; ++ci) cpOf[cpIndices[ci]] = ci;
    constexpr size_t K = 4;
    cpWeights.resize(nv);
    std::vector<std::pair<double, uint32_t>> near;
    near.reserve(nc);
    for (uint32_t v = 0; v < nv; ++v) {
        auto it = cpOf.find(v);
        if (it != cpOf.end()) {
            cpWeights[v].push_back({it->second, 1.0});
            continue;
        }
        near.clear();
        for (uint32_t ci = 0; ci < nc; ++ci) near.push_back({dist(pos[cpIndices[ci]], pos[v]), ci});
        size_t keep = std::min(K, near.size());
        std::partial_sort(near.begin(), near.begin() + keep, near.end());
        const double eps = 1e-12;
        double total = 0.0;
        for (size_t j = 0; j < keep; ++j) total += 1.0 / std::max(near[j].first, eps);
        for (size_t j = 0; j < keep; ++j)
            cpWeights[v].push_back({near[j].second, (1.0 / std::max(near[j].first, eps)) / total});
    }
    return nc;
}

// SurfaceMesh::setControlPointStride regular-grid path, surface_mesh.cpp:319-431
// (N x N vertex grids): every stride-th grid vertex of the interior plus the
// interior's last row/column are control points; the rest are bilinear.
uint32_t Mesh::setControlPointStrideGrid(int stride) {
    cpStride = stride;
    cpIndices.clear();
    cpWeights.clear();
    if (stride <= 0) return 0;
    uint32_t nv = vertexCount();
    int full = static_cast<int>(std::sqrt(static_cast<double>(nv)));
    if (full * full != static_cast<int>(nv) || full < 2) {
        cpStride = 0;  // unstructured meshes use LithologyModelHost::setControlPointStride
        return 0;
    }
    int i0 = paddingRings, i1 = full - paddingRings - 1;
    std::vector<bool> isCP(nv, false);
    for (int r = i0; r <= i1; ++r) {
        int ri = ((r - i0) / stride) * stride + i0;
        if (ri > i1) ri = i1;
        if (r != ri && r != i0 && r != i1) continue;
        for (int c = i0; c <= i1; ++c) {
            int ci = ((c - i0) / stride) * stride + i0;
            if (ci > i1) ci = i1;
            if (c != ci && c != i0 && c != i1) continue;
            isCP[static_cast<size_t>(r * full + c)] = true;
        }
    }
    std::vector<int> cpOf(nv, -1);
    for (uint32_t v = 0; v < nv; ++v)
        if (isCP[v]) {
            cpOf[v] = static_cast<int>(cpIndices.size());
            cpIndices.push_back(v);
        }
    cpWeights.resize(nv);
    for (uint32_t v = 0; v < nv; ++v) {
        if (isCP[v]) {
            cpWeights[v].push_back({static_cast<uint32_t>(cpOf[v]), 1.0});
            continue;
        }
        int r = static_cast<int>(v) / full, c = static_cast<int>(v) % full;
        int r0, r1, c0, c1;
        if (r < i0) { r0 = r1 = i0; } else if (r > i1) { r0 = r1 = i1; } else {
            r0 = ((r - i0) / stride) * stride + i0;
            r1 = std::min(r0 + stride, i1);
        }
        if (c < i0) { c0 = c1 = i0; } else if (c > i1) { c0 = c1 = i1; } else {
            c0 = ((c - i0) / stride) * stride + i0;
            c1 = std::min(c0 + stride, i1);
        }
        double dr = (r1 > r0) ? double(r - r0) / double(r1 - r0) : 0.0;
        double dc = (c1 > c0) ? double(c - c0) / double(c1 - c0) : 0.0;
        auto add = [&](int rr, int cc, double w) {
            if (w < 1e-15) return;
            int cp = cpOf[static_cast<size_t>(rr * full + cc)];
            if (cp >= 0) cpWeights[v].push_back({static_cast<uint32_t>(cp), w});
        };
        add(r0, c0, (1.0 - dr) * (1.0 - dc));
        add(r0, c1, (1.0 - dr) * dc);
        add(r1, c0, dr * (1.0 - dc));
        add(r1, c1, dr * dc);
    }
    return static_cast<uint32_t>(cpIndices.size());
}

// LithologyModel::addGroup, lithology_model.cpp:17-28 (the reference also
// rejects density <= 0 through LithoGroup::isValid; this host model accepts
// any density contrast, which callers of the reference set after adding).
int LithologyModelHost::addGroup(const Group& g) {
    for (auto& e : groups_)
        if (e.id == g.id) return -1;
    groups_.push_back(g);
    dofsDirty_ = true;
    return static_cast<int>(groups_.size()) - 1;
}

int LithologyModelHost::setGroupMesh(int group, Mesh mesh) {
    if (group < 0) return -1;
    if (static_cast<size_t>(group) >= meshes_.size()) {
        meshes_.resize(group + 1);
        hasMesh_.resize(group + 1, 0);
    }
    mesh.rebuildDofMappings();
    meshes_[group] = std::move(mesh);
    hasMesh_[group] = 1;
    dofsDirty_ = true;
    return 0;
}

// LithologyModel::rebuildGlobalDofs, lithology_model.cpp:113-168: DOFs at the
// same micrometre-quantised position and axis share one global DOF.  The
// XOR-shift key is reproduced exactly (it can alias distinct positions, and
// the reference then merges them too).
void LithologyModelHost::rebuildGlobalDofs() {
    globalRefs_.clear();
    std::unordered_map<uint64_t, size_t> keyToGlobal;
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi]) continue;
        const Mesh& m = meshes_[mi];
        for (uint32_t li = 0; li < m.dofs.size(); ++li) {
            const DofMapping& dm = m.dofs[li];
            const Vec3& p = m.pos[dm.vertex];
            uint64_t k = static_cast<uint64_t>(quantize(p.x));
            k ^= (static_cast<uint64_t>(quantize(p.y)) << 21);
            k ^= (static_cast<uint64_t>(quantize(p.z)) << 42);
            k ^= (static_cast<uint64_t>(dm.axis) << 60);
            auto it = keyToGlobal.find(k);
            if (it == keyToGlobal.end()) {
                keyToGlobal[k] = globalRefs_.size();
                globalRefs_.push_back({{static_cast<uint32_t>(mi), li}});
            } else {
                globalRefs_[it->second].push_back({static_cast<uint32_t>(mi), li});
            }
        }
    }
    dofsDirty_ = false;
}

uint32_t LithologyModelHost::totalDofCount() {
    if (dofsDirty_) rebuildGlobalDofs();
    return static_cast<uint32_t>(globalRefs_.size());
}

// LithologyModel::assembleParameterVector, lithology_model.cpp:194-208.
std::vector<double> LithologyModelHost::assembleParameterVector() {
    if (dofsDirty_) rebuildGlobalDofs();
    std::vector<double> p(globalRefs_.size());
    for (size_t g = 0; g < globalRefs_.size(); ++g) {
        const Ref& r = globalRefs_[g][0];
        const Mesh& m = meshes_[r.mesh];
        const DofMapping& dm = m.dofs[r.local];
        p[g] = m.pos[dm.vertex][dm.axis] / m.axisScale[dm.axis];
    }
    return p;
}

// LithologyModel::getBounds, lithology_model.cpp:250-282.
void LithologyModelHost::getBounds(std::vector<double>& lo, std::vector<double>& hi) {
    if (dofsDirty_) rebuildGlobalDofs();
    lo.assign(globalRefs_.size(), -1e12);
    hi.assign(globalRefs_.size(), 1e12);
    for (size_t g = 0; g < globalRefs_.size(); ++g) {
        double l = -1e12, h = 1e12;
        for (const Ref& r : globalRefs_[g]) {
            const Mesh& m = meshes_[r.mesh];
            const DofMapping& dm = m.dofs[r.local];
            double s = m.axisScale[dm.axis];
            if (dm.axis == 2) {
                l = std::max(l, m.minDepth / s);
                h = std::min(h, m.maxDepth / s);
            } else if (dm.axis == 0) {
                l = std::max(l, boundsMin_.x / s);
                h = std::min(h, boundsMax_.x / s);
            } else {
                l = std::max(l, boundsMin_.y / s);
                h = std::min(h, boundsMax_.y / s);
            }
        }
        lo[g] = l;
        hi[g] = h;
    }
}

// LithologyModel::applyModelBounds, lithology_model.cpp:808-850.
void LithologyModelHost::applyModelBounds(double marginMultiplier) {
    if (meshes_.empty()) return;
    double mn[3] = {1e30, 1e30, 1e30}, mx[3] = {-1e30, -1e30, -1e30};
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi]) continue;
        for (const Vec3& p : meshes_[mi].pos)
            for (int k = 0; k < 3; ++k) {
                if (p[k] < mn[k]) mn[k] = p[k];
                if (p[k] > mx[k]) mx[k] = p[k];
            }
    }
    double margin = std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2], 1.0}) * 0.01 * marginMultiplier;
    boundsMin_ = {mn[0] - margin, mn[1] - margin, mn[2] - margin};
    boundsMax_ = {mx[0] + margin, mx[1] + margin, mx[2] + margin};
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi]) continue;
        meshes_[mi].minDepth = mn[2] - margin;
        meshes_[mi].maxDepth = mx[2] + margin;
    }
    dofsDirty_ = true;
}

// LithologyModel::buildSharedVertexSync, lithology_model.cpp:585-618.
void LithologyModelHost::buildSharedVertexSync() {
    if (meshes_.size() < 2) return;
    std::map<PosKey, std::vector<Ref>> byPos;
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi]) continue;
        const Mesh& m = meshes_[mi];
        for (uint32_t v = 0; v < m.vertexCount(); ++v)
            byPos[{quantize(m.pos[v].x), quantize(m.pos[v].y), quantize(m.pos[v].z)}].push_back(
                {static_cast<uint32_t>(mi), v});
    }
    sharedSync_.clear();
    for (auto& kv : byPos)
        if (kv.second.size() >= 2) sharedSync_.push_back(std::move(kv.second));
}

// LithologyModel::setControlPointStride, lithology_model.cpp:864-1040:
// mesh-independent control points on a common lattice of `stride` cells, one
// per populated cell (the position closest to the cell centre); shared
// positions make every owning mesh carry the control point.
uint32_t LithologyModelHost::setControlPointStride(int stride) {
    cpStride_ = stride;
    dofsDirty_ = true;
    if (stride <= 0) {
        for (size_t mi = 0; mi < meshes_.size(); ++mi) {
            if (!hasMesh_[mi]) continue;
            meshes_[mi].cpStride = 0;
            meshes_[mi].cpIndices.clear();
            meshes_[mi].cpWeights.clear();
            meshes_[mi].rebuildDofMappings();
        }
        return totalDofCount();
    }
    std::map<PosKey, std::vector<std::pair<uint32_t, uint32_t>>> byPos;
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi]) continue;
        const Mesh& m = meshes_[mi];
        for (uint32_t v = 0; v < m.vertexCount(); ++v)
            byPos[{quantize(m.pos[v].x), quantize(m.pos[v].y), quantize(m.pos[v].z)}].push_back(
                {static_cast<uint32_t>(mi), v});
    }
    if (byPos.size() < 4) {
        cpStride_ = 0;
        return 0;
    }
    double minD[3] = {1e12, 1e12, 1e12};
    {
        std::vector<PosKey> keys;
        keys.reserve(byPos.size());
        for (const auto& kv : byPos) keys.push_back(kv.first);
        size_t n = std::min(keys.size(), size_t(300));
        for (size_t i = 0; i < n; ++i)
            for (size_t j = i + 1; j < n; ++j) {
                double d[3] = {std::abs(static_cast<double>(keys[i].x - keys[j].x)) * 1e-6,
                               std::abs(static_cast<double>(keys[i].y - keys[j].y)) * 1e-6,
                               std::abs(static_cast<double>(keys[i].z - keys[j].z)) * 1e-6};
                for (int k = 0; k < 3; ++k)
                    if (d[k] > 0 && d[k] < minD[k]) minD[k] = d[k];
            }
    }
    double cell = std::max({minD[0], minD[1], minD[2], 1.0});
    double cellQ = cell * 1e6;
    int64_t strideQ = static_cast<int64_t>(stride) * static_cast<int64_t>(cellQ);
    if (strideQ < 1) strideQ = 1;
    auto gridCell = [strideQ](int64_t q) -> int64_t { return q >= 0 ? q / strideQ : (q - strideQ + 1) / strideQ; };
    struct Best { PosKey pos; int64_t d2; };
    std::map<PosKey, Best> cellBest;  // keyed by cell coordinates
    for (const auto& kv : byPos) {
        const PosKey& k = kv.first;
        PosKey ck{gridCell(k.x), gridCell(k.y), gridCell(k.z)};
        int64_t cx = ck.x * strideQ + strideQ / 2, cy = ck.y * strideQ + strideQ / 2, cz = ck.z * strideQ + strideQ / 2;
        int64_t d2 = (k.x - cx) * (k.x - cx) + (k.y - cy) * (k.y - cy) + (k.z - cz) * (k.z - cz);
        auto it = cellBest.find(ck);
        if (it == cellBest.end()) cellBest[ck] = {k, d2};
        else if (d2 < it->second.d2) it->second = {k, d2};
    }
    std::set<PosKey> cpPos;
    for (const auto& kv : cellBest) cpPos.insert(kv.second.pos);
    std::vector<std::vector<uint32_t>> meshCPs(meshes_.size());
    for (const PosKey& pk : cpPos) {
        auto it = byPos.find(pk);
        if (it == byPos.end()) continue;
        for (const auto& mv : it->second) meshCPs[mv.first].push_back(mv.second);
    }
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi] || meshCPs[mi].empty()) continue;
        meshes_[mi].setControlPointsExplicit(meshCPs[mi]);
        meshes_[mi].rebuildDofMappings();
    }
    buildSharedVertexSync();
    return totalDofCount();
}

// LithologyModel::applyParameterVector, lithology_model.cpp:210-248 (host
// copy, used by tests and by the host-side model state after an inversion).
void LithologyModelHost::applyParameterVector(const std::vector<double>& params) {
    if (dofsDirty_) rebuildGlobalDofs();
    for (size_t g = 0; g < globalRefs_.size(); ++g)
        for (const Ref& r : globalRefs_[g]) {
            Mesh& m = meshes_[r.mesh];
            const DofMapping& dm = m.dofs[r.local];
            m.pos[dm.vertex][dm.axis] = params[g] * m.axisScale[dm.axis];
        }
    for (size_t mi = 0; mi < meshes_.size(); ++mi) {
        if (!hasMesh_[mi]) continue;
        Mesh& m = meshes_[mi];
        if (m.cpStride <= 0) continue;
        for (uint32_t v = 0; v < m.vertexCount(); ++v) {
            if (m.isControlPoint(v)) continue;
            Vec3 p;
            for (const auto& cw : m.cpWeights[v]) {
                const Vec3& q = m.pos[m.cpIndices[cw.first]];
                p.x += cw.second * q.x; p.y += cw.second * q.y; p.z += cw.second * q.z;
            }
            m.pos[v] = p;
        }
    }
    for (const auto& grp : sharedSync_) {
        if (grp.size() < 2) continue;
        Vec3 a;
        for (const Ref& r : grp) {
            const Vec3& q = meshes_[r.mesh].pos[r.local];
            a.x += q.x; a.y += q.y; a.z += q.z;
        }
        double n = static_cast<double>(grp.size());
        a.x /= n; a.y /= n; a.z /= n;
        for (const Ref& r : grp) meshes_[r.mesh].pos[r.local] = a;
    }
}

ModelTables LithologyModelHost::tables() {
    if (dofsDirty_) rebuildGlobalDofs();
    ModelTables t;
    int G = static_cast<int>(groups_.size());
    t.nGroups = G;
    t.vertexOffset.assign(G + 1, 0);
    t.grpTriOff.assign(G + 1, 0);
    std::vector<int32_t> meshBase(meshes_.size(), 0);
    int v = 0, tcount = 0;
    for (int g = 0; g < G; ++g) {
        t.vertexOffset[g] = v;
        t.grpTriOff[g] = tcount;
        if (const Mesh* m = mesh(g)) {
            meshBase[g] = v;
            for (const Vec3& p : m->pos) { t.pos.push_back(p.x); t.pos.push_back(p.y); t.pos.push_back(p.z); }
            for (uint32_t x : m->tri) t.tri.push_back(static_cast<int32_t>(x) + v);
            v += static_cast<int>(m->vertexCount());
            tcount += static_cast<int>(m->triangleCount());
        }
    }
    t.vertexOffset[G] = v;
    t.grpTriOff[G] = tcount;
    t.nVertices = v;
    t.nTriangles = tcount;
    t.nDofs = static_cast<int>(globalRefs_.size());
    t.dofOff.push_back(0);
    for (const auto& refs : globalRefs_) {
        for (const Ref& r : refs) {
            const Mesh& m = meshes_[r.mesh];
            const DofMapping& dm = m.dofs[r.local];
            t.refVertex.push_back(meshBase[r.mesh] + static_cast<int32_t>(dm.vertex));
            t.refAxis.push_back(dm.axis);
            t.refScale.push_back(m.axisScale[dm.axis]);
        }
        t.dofOff.push_back(static_cast<int32_t>(t.refVertex.size()));
    }
    t.interpOff.assign(v + 1, 0);
    for (int g = 0; g < G; ++g) {
        const Mesh* m = mesh(g);
        for (uint32_t lv = 0; m && lv < m->vertexCount(); ++lv) {
            int gv = meshBase[g] + static_cast<int>(lv);
            t.interpOff[gv] = static_cast<int32_t>(t.interpSrc.size());
            if (m->cpStride <= 0 || m->isControlPoint(lv)) continue;
            for (const auto& cw : m->cpWeights[lv]) {
                t.interpSrc.push_back(meshBase[g] + static_cast<int32_t>(m->cpIndices[cw.first]));
                t.interpW.push_back(cw.second);
            }
        }
    }
    // rows were opened in vertex order, so row i ends where row i+1 starts
    t.interpOff[v] = static_cast<int32_t>(t.interpSrc.size());
    t.syncOff.push_back(0);
    for (const auto& grp : sharedSync_) {
        for (const Ref& r : grp) t.syncVertex.push_back(meshBase[r.mesh] + static_cast<int32_t>(r.local));
        t.syncOff.push_back(static_cast<int32_t>(t.syncVertex.size()));
    }
    return t;
}

}  // namespace litho_b200
