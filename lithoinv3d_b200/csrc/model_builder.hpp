// Host-side lithology model: groups, one closed triangulated mesh per group,
// vertex freedoms, per-mesh DOF mappings, global DOF de-duplication,
// control-point selection/interpolation and shared-vertex synchronisation.
//
// This is setup-time bookkeeping; it produces the flat tables the device path
// consumes (lf_set_model).  Semantics follow the reference's SurfaceMesh
// (modules/litho-surface/src/surface/surface_mesh.cpp) and LithologyModel
// (modules/litho-model/src/litho/lithology_model.cpp), cited per function in
// model_builder.cpp.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace litho_b200 {

// VertexFreedom numbering, modules/litho-surface/include/litho_invert/surface/surface_mesh.h:9-19.
enum Freedom : uint8_t {
    FIXED = 0, Z_ONLY, X_ONLY, Y_ONLY, ALONG_VECTOR, XY_FREE, XZ_FREE, YZ_FREE, XYZ_FREE
};

struct Vec3 {
    double x = 0, y = 0, z = 0;
    double& operator[](int k) { return k == 0 ? x : (k == 1 ? y : z); }
    double operator[](int k) const { return k == 0 ? x : (k == 1 ? y : z); }
};

struct DofMapping {
    uint32_t vertex = 0;
    uint8_t axis = 0;
};

struct Mesh {
    std::vector<Vec3> pos;
    std::vector<uint8_t> freedom;
    std::vector<uint32_t> tri;  // 3 per triangle, mesh-local indices
    double axisScale[3] = {1.0, 1.0, 1.0};
    double minDepth = -10000.0, maxDepth = 0.0;
    int interiorGridDim = 0, paddingRings = 0;
    int cpStride = 0;
    std::vector<uint32_t> cpIndices;
    std::vector<std::vector<std::pair<uint32_t, double>>> cpWeights;
    std::vector<DofMapping> dofs;

    uint32_t vertexCount() const { return static_cast<uint32_t>(pos.size()); }
    uint32_t triangleCount() const { return static_cast<uint32_t>(tri.size() / 3); }
    bool isPadding(uint32_t v) const;
    bool isControlPoint(uint32_t v) const;
    void rebuildDofMappings();
    uint32_t setControlPointsExplicit(const std::vector<uint32_t>& cps);
    uint32_t setControlPointStrideGrid(int stride);
};

struct Group {
    int id = -1;
    double density = 0.0, susceptibility = 0.0;
    double remMagnitude = 0.0, remInclination = 0.0, remDeclination = 0.0;
    Vec3 remVector;
};

// Flat tables for the device (all vertex indices are global: the vertices of
// mesh g occupy [vertexOffset[g], vertexOffset[g+1])).
struct ModelTables {
    int nGroups = 0, nVertices = 0, nTriangles = 0, nDofs = 0;
    std::vector<double> pos;              // V*3
    std::vector<int32_t> tri;             // T*3
    std::vector<int32_t> grpTriOff;       // G+1
    std::vector<int32_t> vertexOffset;    // G+1
    std::vector<int32_t> dofOff;          // np+1
    std::vector<int32_t> refVertex;       // nref
    std::vector<uint8_t> refAxis;         // nref
    std::vector<double> refScale;         // nref
    std::vector<int32_t> interpOff;       // V+1
    std::vector<int32_t> interpSrc;
    std::vector<double> interpW;
    std::vector<int32_t> syncOff;         // ns+1
    std::vector<int32_t> syncVertex;
};

class LithologyModelHost {
public:
    int addGroup(const Group& g);  // -1 if the id already exists
    int setGroupMesh(int group, Mesh mesh);
    int groupCount() const { return static_cast<int>(groups_.size()); }
    Group& group(int g) { return groups_.at(g); }
    const Group& group(int g) const { return groups_.at(g); }
    Mesh* mesh(int g) { return g >= 0 && g < (int)meshes_.size() && hasMesh_[g] ? &meshes_[g] : nullptr; }
    const Mesh* mesh(int g) const { return g >= 0 && g < (int)meshes_.size() && hasMesh_[g] ? &meshes_[g] : nullptr; }
    int meshCount() const { return static_cast<int>(meshes_.size()); }

    uint32_t setControlPointStride(int stride);
    void buildSharedVertexSync();
    void applyModelBounds(double marginMultiplier);

    uint32_t totalDofCount();
    std::vector<double> assembleParameterVector();
    void getBounds(std::vector<double>& lo, std::vector<double>& hi);
    void applyParameterVector(const std::vector<double>& params);  // host reference of the scatter
    ModelTables tables();

    void markDirty() { dofsDirty_ = true; }

private:
    struct Ref { uint32_t mesh, local; };
    std::vector<Group> groups_;
    std::vector<Mesh> meshes_;
    std::vector<uint8_t> hasMesh_;
    std::vector<std::vector<Ref>> globalRefs_;
    std::vector<std::vector<Ref>> sharedSync_;  // (mesh, vertex)
    bool dofsDirty_ = true;
    int cpStride_ = 0;
    Vec3 boundsMin_{-1e12, -1e12, -1e12}, boundsMax_{1e12, 1e12, 1e12};
    void rebuildGlobalDofs();
};

}  // namespace litho_b200
