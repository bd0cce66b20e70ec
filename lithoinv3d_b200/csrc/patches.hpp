// Facet patches of the mixed-precision forward.
//
// The reference evaluates every (station, facet) pair from scratch: per facet
// it recomputes the three vertex distances and the three edge line integrals
// (faceNagyContribution gravity_forward.cpp:13-42 calling lineIntegralTerm
// geometry.cpp:32-52 per edge and solidAngle geometry.cpp:10-30; the same for
// magneticFacet magnetic_forward.cpp:312-347).  On a closed triangulated
// surface a vertex is shared by ~6 facets and an edge by 2, and the edge line
// integral is symmetric in its end points, so a station-tile kernel that walks
// a compact group of facets (a patch) can evaluate each vertex distance and
// each edge integral once per station instead.
//
// A patch is up to kPatchFacets facets of one lithology group whose corners
// are at most kPatchVerts distinct vertices; its edges are the distinct
// (unordered) vertex pairs of its facets, each listing the (at most two)
// facets of the patch that use it -- a third or fourth user of one edge (a
// non-manifold voxel edge) gets a duplicate edge entry.  Patches are grown
// greedily over shared vertices from seeds in Morton order of the facet
// centroids, preferring the candidate facet that adds the fewest new
// vertices, so that patches are compact and share most of their vertices.
//
// Topology only: built once per model (positions change every evaluation,
// the patch membership does not).
#pragma once
#include <cstdint>
#include <vector>

namespace litho_b200 {

constexpr int kPatchFacets = 32;  // one facet per lane in the per-warp near/far test
constexpr int kPatchVerts = 32;   // per-station vertex distances kept in shared memory
constexpr int kPatchEdges = 3 * kPatchFacets;
constexpr int kNoFacet = 255;
// Byte sizes of the per-evaluation records of one patch blob (the device
// structs in kernels_patch.cuh assert the same sizes): header, vertex, edge
// (two records), facet.
constexpr int kPatchHeadBytes = 48;
constexpr int kPatchVertBytes = 16;
constexpr int kPatchEdgeBytes = 32;
constexpr int kPatchFacetBytes = 176;
constexpr int kPatchMaxBytes = kPatchHeadBytes + kPatchVerts * kPatchVertBytes + kPatchEdges * kPatchEdgeBytes +
                               kPatchFacets * kPatchFacetBytes;

struct PatchTopology {
    int P = 0;
    std::vector<int32_t> grpPatchOff;    // [G + 1]: patches of group g
    std::vector<int32_t> facetOff;       // [P + 1] into facets / facetCorners
    std::vector<int32_t> facets;         // global facet index
    std::vector<uint32_t> facetCorners;  // local vertex indices a | b << 8 | c << 16 (the facet's own order)
    std::vector<int32_t> vertOff;        // [P + 1] into verts
    std::vector<int32_t> verts;          // global vertex index
    std::vector<int32_t> edgeOff;        // [P + 1] into edgeInfo
    // lv1 | lv2 << 8 | lf1 << 16 | lf2 << 24 with (lf, i) the patch facet using
    // the edge and the edge's index i (v_i -> v_{i+1}) in that facet;
    // edgeSlot = i1 | i2 << 2; lf2 == kNoFacet when one facet uses the edge
    std::vector<uint32_t> edgeInfo;
    std::vector<uint8_t> edgeSlot;
    std::vector<int32_t> blobOff;  // [P + 1] byte offset of each patch's record blob
};

// tri[3 * nt] (global vertex indices), grpTriOff[G + 1], xyz[3 * nv]
// (positions used only for the seed order).
PatchTopology build_patches(int nv, const double* xyz, int nt, const int32_t* tri, int G, const int32_t* grpTriOff);

}  // namespace litho_b200
