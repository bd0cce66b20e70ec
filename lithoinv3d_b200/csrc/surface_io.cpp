// Surface files on either side of the path: the GOCAD TSurf and OBJ readers
// of the reference (loadSurfaceMesh / TSurfaceLoader::load /
// OBJSurfaceLoader::load, modules/litho-io/src/io/surface_loader.cpp:9-181)
// and its TSurf writer (InversionExporter::exportTS,
// modules/litho-io/src/io/exporters.cpp:116-151), as plain C-ABI functions.
// The readers tokenise with the same stream extraction as the reference, so
// coordinates parse to the same doubles; unlike the reference they reject a
// triangle whose vertex index falls outside the file's vertices instead of
// returning a mesh that would fault later.
#include "../../include/litho_gpu.h"

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct SurfaceData {
    std::vector<double> xyz;
    std::vector<int64_t> tri;  // 0-based, as read (checked afterwards)
};

// TSurfaceLoader::load (surface_loader.cpp:93-161)
bool read_tsurf(const std::string& path, SurfaceData& s) {
    std::ifstream file(path);
    if (!file.is_open()) return false;
    std::string line;
    bool inHeader = false;
    while (std::getline(file, line)) {
        const size_t start = line.find_first_not_of(" \t\r");
        if (start == std::string::npos) continue;
        line = line.substr(start);
        if (line.empty() || line[0] == '#') continue;
        if (inHeader) {
            if (line[0] == '}') inHeader = false;
            continue;
        }
        if (line.find("HEADER") != std::string::npos && line.find('{') != std::string::npos) {
            inHeader = true;
            continue;
        }
        if (line == "END") break;
        if (line == "TFACE" || line == "TRIANGLES") continue;
        if (line.rfind("GOCAD", 0) == 0) continue;
        std::stringstream ss(line);
        std::string keyword;
        ss >> keyword;
        if (keyword == "VRTX" || keyword == "PVRTX") {
            int idx;
            double x, y, z;
            if (!(ss >> idx >> x >> y >> z)) continue;  // malformed vertex line: skipped, as the reference does
            s.xyz.push_back(x);
            s.xyz.push_back(y);
            s.xyz.push_back(z);
        } else if (keyword == "TRGL") {
            int v1, v2, v3;
            if (!(ss >> v1 >> v2 >> v3)) continue;
            s.tri.push_back((int64_t)v1 - 1);
            s.tri.push_back((int64_t)v2 - 1);
            s.tri.push_back((int64_t)v3 - 1);
        }
    }
    return !s.xyz.empty();
}

// OBJSurfaceLoader::load (surface_loader.cpp:9-91): "v x y z" vertices,
// "f" / "fo" faces with 1-based indices (the part before the first '/'),
// polygons fanned from their first vertex.
bool read_obj(const std::string& path, SurfaceData& s) {
    std::ifstream file(path);
    if (!file.is_open()) return false;
    std::string line;
    while (std::getline(file, line)) {
        const size_t start = line.find_first_not_of(" \t\r");
        if (start == std::string::npos) continue;
        line = line.substr(start);
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ss(line);
        std::string keyword;
        ss >> keyword;
        if (keyword == "v") {
            double x, y, z;
            if (!(ss >> x >> y >> z)) continue;
            s.xyz.push_back(x);
            s.xyz.push_back(y);
            s.xyz.push_back(z);
        } else if (keyword == "f" || keyword == "fo") {
            std::vector<int> idx;
            std::string token;
            bool bad = false;
            while (ss >> token) {
                const size_t slash = token.find('/');
                if (slash != std::string::npos) token = token.substr(0, slash);
                try {
                    idx.push_back(std::stoi(token));
                } catch (...) {
                    bad = true;
                    break;
                }
            }
            if (bad || idx.size() < 3) continue;
            for (size_t i = 1; i + 1 < idx.size(); ++i) {
                s.tri.push_back((int64_t)idx[0] - 1);
                s.tri.push_back((int64_t)idx[i] - 1);
                s.tri.push_back((int64_t)idx[i + 1] - 1);
            }
        }
    }
    return !s.xyz.empty();
}

}  // namespace

extern "C" lf_status lf_read_surface(const char* path, int* n_vertices, int* n_triangles, double* xyz,
                                     int32_t* tri) {
    if (!path || !n_vertices || !n_triangles) return LF_EINVAL;
    std::string p(path), ext;
    const size_t dot = p.rfind('.');
    if (dot != std::string::npos) {
        ext = p.substr(dot);
        for (auto& ch : ext) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    }
    SurfaceData s;
    bool ok = false;
    if (ext == ".ts") ok = read_tsurf(p, s);
    else if (ext == ".obj") ok = read_obj(p, s);
    else return LF_EINVAL;  // loadSurfaceMesh: unrecognised extension
    if (!ok) return LF_EINVAL;  // unreadable, or no vertices
    const int64_t nv = (int64_t)s.xyz.size() / 3, nt = (int64_t)s.tri.size() / 3;
    if (nv > INT32_MAX || nt > INT32_MAX) return LF_EINVAL;
    for (int64_t v : s.tri)
        if (v < 0 || v >= nv) return LF_EINVAL;  // triangle names a vertex the file does not have
    *n_vertices = static_cast<int>(nv);
    *n_triangles = static_cast<int>(nt);
    if (xyz)
        for (size_t i = 0; i < s.xyz.size(); ++i) xyz[i] = s.xyz[i];
    if (tri)
        for (size_t i = 0; i < s.tri.size(); ++i) tri[i] = static_cast<int32_t>(s.tri[i]);
    return LF_OK;
}

extern "C" lf_status lf_write_tsurf(const char* path, const char* name, int n_vertices, const double* xyz,
                                    int n_triangles, const int32_t* tri) {
    if (!path || !name || n_vertices < 0 || n_triangles < 0 || (n_vertices > 0 && !xyz) ||
        (n_triangles > 0 && !tri))
        return LF_EINVAL;
    for (int64_t i = 0; i < 3 * (int64_t)n_triangles; ++i)
        if (tri[i] < 0 || tri[i] >= n_vertices) return LF_EINVAL;
    std::ofstream out(path);
    if (!out.is_open()) return LF_EINVAL;
    out << "GOCAD TSurf 1\n";
    out << "HEADER {\n";
    out << "  name: " << name << "\n";
    out << "}\n";
    out << "TFACE\n";
    for (int i = 0; i < n_vertices; ++i)
        out << "VRTX " << (i + 1) << " " << std::scientific << std::setprecision(8) << xyz[3 * i] << " "
            << xyz[3 * i + 1] << " " << xyz[3 * i + 2] << "\n";
    for (int i = 0; i < n_triangles; ++i)
        out << "TRGL " << (tri[3 * i] + 1) << " " << (tri[3 * i + 1] + 1) << " " << (tri[3 * i + 2] + 1) << "\n";
    out << "END\n";
    return out.good() ? LF_OK : LF_EINVAL;
}
