// Host-side file formats: the STL reader (src/geom/stl_loader.cpp:34-122) and
// the ASCII legacy-VTK writers (src/moment_vtk_writer.cu:9-49).  The VTK
// header lines and the value formatting (operator<< on float, 6 significant
// digits) are kept identical so existing post-processing (ParaView, the
// reference's scripts/vtk_slice_to_png.py) reads the files unchanged.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "lbm_capi.h"

namespace lbm {
void set_error(const std::string& msg);
int write_vtk_file(int kind, const float* a, const float* b, const float* c, int nx, int ny, int nz, const char* path);
}

namespace {

void bb_add(float* bb, const float* p) {
    for (int k = 0; k < 3; ++k) {
        if (p[k] < bb[k]) bb[k] = p[k];
        if (bb[3 + k] < p[k]) bb[3 + k] = p[k];
    }
}

void bb_reset(float* bb) {
    for (int k = 0; k < 3; ++k) { bb[k] = FLT_MAX; bb[3 + k] = -FLT_MAX; }
}

// ASCII: every "vertex x y z" line adds a vertex; three make a triangle.
bool parse_ascii(const std::string& s, std::vector<float>& t, float* bb) {
    bb_reset(bb);
    t.clear();
    std::istringstream is(s);
    std::string line;
    float tri[9];
    int nv = 0;
    while (std::getline(is, line)) {
        std::istringstream ls(line);
        std::string tok;
        ls >> tok;
        if (tok != "vertex") continue;
        float x = 0, y = 0, z = 0;
        ls >> x >> y >> z;
        tri[nv * 3 + 0] = x; tri[nv * 3 + 1] = y; tri[nv * 3 + 2] = z;
        if (++nv == 3) {
            t.insert(t.end(), tri, tri + 9);
            for (int v = 0; v < 3; ++v) bb_add(bb, tri + v * 3);
            nv = 0;
        }
    }
    return !t.empty();
}

// Binary: 80-byte header, uint32 count, 50-byte records (normal, 3 vertices, attribute).
bool parse_binary(const std::string& s, std::vector<float>& t, float* bb) {
    bb_reset(bb);
    t.clear();
    if (s.size() < 84) return false;
    uint32_t n = 0;
    std::memcpy(&n, s.data() + 80, 4);
    if ((uint64_t)84 + (uint64_t)n * 50u > (uint64_t)s.size()) return false;
    t.resize((size_t)n * 9);
    for (uint32_t i = 0; i < n; ++i) {
        std::memcpy(&t[(size_t)i * 9], s.data() + 84 + (size_t)i * 50 + 12, 36);
        for (int v = 0; v < 3; ++v) bb_add(bb, &t[(size_t)i * 9 + v * 3]);
    }
    return true;
}

std::string read_all(const char* path, bool& ok) {
    std::ifstream f(path, std::ios::binary);
    ok = static_cast<bool>(f);
    if (!ok) return {};
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}


}  // namespace

extern "C" {

int lbm_load_stl(const char* path, float** tris, int64_t* ntri, float* bb) {
    if (!path || !tris || !ntri || !bb) { lbm::set_error("lbm_load_stl: null argument"); return LBM_ERR_INVALID; }
    bool ok = false;
    const std::string s = read_all(path, ok);
    if (!ok) { lbm::set_error(std::string("cannot open STL: ") + path); return LBM_ERR_IO; }
    std::vector<float> t;
    bool good;
    if (s.size() >= 5 && s.compare(0, 5, "solid") == 0) {
        good = parse_ascii(s, t, bb);
        if (!good) good = parse_binary(s, t, bb);
    } else {
        good = parse_binary(s, t, bb);
    }
    if (!good) { lbm::set_error(std::string("malformed STL: ") + path); return LBM_ERR_IO; }
    float* out = static_cast<float*>(std::malloc(sizeof(float) * (t.empty() ? 1 : t.size())));
    if (!out) { lbm::set_error("lbm_load_stl: out of host memory"); return LBM_ERR_ALLOC; }
    if (!t.empty()) std::memcpy(out, t.data(), sizeof(float) * t.size());
    *tris = out;
    *ntri = (int64_t)(t.size() / 9);
    return LBM_OK;
}

void lbm_free(void* p) { std::free(p); }

// The text is formatted on the GPU (lbm_vtk.cu), byte-identical to the
// reference's `ofstream << float` writer (src/moment_vtk_writer.cu:8-48).
int lbm_write_scalar_vtk(const char* filename, const float* d_field, int Nx, int Ny, int Nz) {
    if (!filename || !d_field) { lbm::set_error("write_scalar_vtk: null argument"); return LBM_ERR_INVALID; }
    return lbm::write_vtk_file(LBM_VTK_SCALAR, d_field, nullptr, nullptr, Nx, Ny, Nz, filename);
}

int lbm_write_vector_vtk(const char* filename, const float* d_fx, const float* d_fy, const float* d_fz, int Nx,
                         int Ny, int Nz) {
    if (!filename || !d_fx || !d_fy || !d_fz) { lbm::set_error("write_vector_vtk: null argument"); return LBM_ERR_INVALID; }
    return lbm::write_vtk_file(LBM_VTK_VECTOR, d_fx, d_fy, d_fz, Nx, Ny, Nz, filename);
}

void write_scalar_vtk(const char* filename, const float* d_field, int Nx, int Ny, int Nz) {
    if (lbm_write_scalar_vtk(filename, d_field, Nx, Ny, Nz) != LBM_OK)
        std::fprintf(stderr, "[vtk] %s\n", lbm_last_error());
}

void write_vector_vtk(const char* filename, const float* d_fx, const float* d_fy, const float* d_fz, int Nx, int Ny,
                      int Nz) {
    if (lbm_write_vector_vtk(filename, d_fx, d_fy, d_fz, Nx, Ny, Nz) != LBM_OK)
        std::fprintf(stderr, "[vtk] %s\n", lbm_last_error());
}

}  // extern "C"
