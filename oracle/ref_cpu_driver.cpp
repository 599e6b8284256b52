// Checker only: a C-ABI around the reference's own CPU geometry code
// (src/geom/stl_loader.cpp, src/geom/voxelize.cpp) and the band BFS in
// src/apps/sim_runner.hpp:28-91, compiled from the reference sources by
// oracle/build_ref.sh into oracle/_ref/libref_cpu.so.  Used by tests to pin
// the oracle and to generate golden masks; never part of the product.
#include <cstdint>
#include <cstring>
#include <vector>

#include "apps/sim_runner.hpp"   // pulls in sim_common.hpp, stl_loader.hpp, voxelize.hpp

extern "C" {

// load_stl (stl_loader.cpp:102-122).  Returns triangle count or -1; positions
// are returned as 9 floats per triangle and bb = {bbmin, bbmax}.
int64_t ref_load_stl(const char* path, float* tris_out, int64_t cap_tris, float* bb) {
    TriangleMesh m;
    if (!load_stl(path, m)) return -1;
    const int64_t ntri = (int64_t)(m.indices.size() / 3);
    bb[0] = m.bbmin.x; bb[1] = m.bbmin.y; bb[2] = m.bbmin.z;
    bb[3] = m.bbmax.x; bb[4] = m.bbmax.y; bb[5] = m.bbmax.z;
    if (tris_out) {
        for (int64_t t = 0; t < ntri && t < cap_tris; ++t)
            for (int v = 0; v < 3; ++v) {
                const glm::vec3& p = m.positions[m.indices[(size_t)t * 3 + v]];
                tris_out[t * 9 + v * 3 + 0] = p.x;
                tris_out[t * 9 + v * 3 + 1] = p.y;
                tris_out[t * 9 + v * 3 + 2] = p.z;
            }
    }
    return ntri;
}

// voxelize_mesh_to_mask (voxelize.cpp:228-243) on an unindexed triangle soup.
int ref_voxelize(const float* tris, int64_t ntri, const float* bb, int nx, int ny, int nz,
                 float scale, float tx, float ty, float tz, int refine, float thr, uint8_t* out) {
    TriangleMesh m;
    m.positions.reserve((size_t)ntri * 3);
    for (int64_t i = 0; i < ntri * 3; ++i) {
        m.positions.emplace_back(tris[i * 3 + 0], tris[i * 3 + 1], tris[i * 3 + 2]);
        m.indices.push_back((unsigned)i);
    }
    m.bbmin = glm::vec3(bb[0], bb[1], bb[2]);
    m.bbmax = glm::vec3(bb[3], bb[4], bb[5]);
    VoxelParams vp;
    vp.Nx = nx; vp.Ny = ny; vp.Nz = nz;
    vp.uniformScale = scale;
    vp.translate = glm::vec3(tx, ty, tz);
    vp.refine = refine;
    vp.coverageThreshold = thr;
    std::vector<unsigned char> mask = voxelize_mesh_to_mask(m, vp);
    std::memcpy(out, mask.data(), mask.size());
    return 0;
}

// build_obstacle (sim_common.hpp:211-238): STL path + CLI voxel options -> mask.
// Returns 1 with an obstacle, 0 without (load failure), as the reference does.
int ref_build_obstacle(const char* stl_path, int nx, int ny, int nz, float scale,
                       float tx, float ty, float tz, int amr_factor, float amr_thr, uint8_t* out) {
    DomainConfig dom; dom.Nx = nx; dom.Ny = ny; dom.Nz = nz;
    ObstacleConfig obs;
    obs.stlPath = stl_path ? stl_path : "";
    obs.uniformScale = scale;
    obs.translateX = tx; obs.translateY = ty; obs.translateZ = tz;
    obs.amrFactor = amr_factor;
    obs.amrThreshold = amr_thr;
    ObstacleData od = build_obstacle(dom, obs);
    std::memcpy(out, od.solidMask.data(), od.solidMask.size());
    return od.hasObstacle ? 1 : 0;
}

// build_distance_to_solid_6n + build_legacy_mask_from_distance, called the
// way run_hybrid_b0 does (sim_runner.hpp:221-224).
void ref_band(const uint8_t* mask, int nx, int ny, int nz, int d0, int32_t* dist_out, uint8_t* legacy_out) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<unsigned char> m(mask, mask + N);
    const int maxDist = std::max(1, d0);
    std::vector<int> dist = build_distance_to_solid_6n(m, nx, ny, nz, maxDist);
    std::vector<unsigned char> leg = build_legacy_mask_from_distance(m, dist, d0);
    for (size_t i = 0; i < N; ++i) { dist_out[i] = dist[i]; legacy_out[i] = leg[i]; }
}

// parse_common_args (sim_common.hpp:115-192) on an argv, printed as the
// key=value lines that the library's command-line tools print with
// --print-config.  Returns the length written, or -1 when the reference's
// parser throws (std::stoi/stof on a non-number).
int ref_parse_common_args(int argc, char** argv, int hybrid, char* out, int cap) {
    DomainConfig dom;
    ObstacleConfig obs;
    RunConfig run;
    HybridConfig hyb;
    try {
        parse_common_args(argc, argv, dom, obs, run, hybrid ? &hyb : nullptr);
    } catch (...) {
        return -1;
    }
    return std::snprintf(
        out, (size_t)cap,
        "nx=%d\nny=%d\nnz=%d\ntau=%.9g\nforce=%.9g,%.9g,%.9g\n"
        "stl=%s\nvoxel_scale=%.9g\nvoxel_translate=%.9g,%.9g,%.9g\namr_factor=%d\namr_threshold=%.9g\n"
        "steps=%d\nsubsteps=%d\nvtk_dir=%s\nvtk_every=%d\ninit=%s\namp=%.9g\nsigma=%.9g\n"
        "center=%.9g,%.9g,%.9g\nslab_axis=%d\nslab_center=%.9g\nslab_width=%.9g\nband_d0=%d\n",
        dom.Nx, dom.Ny, dom.Nz, dom.tau, dom.fx, dom.fy, dom.fz, obs.stlPath.c_str(), obs.uniformScale,
        obs.translateX, obs.translateY, obs.translateZ, obs.amrFactor, obs.amrThreshold, run.steps, run.substeps,
        run.vtkDir.c_str(), run.vtkEvery, run.initMode.c_str(), run.amp, run.sigma, run.cx, run.cy, run.cz,
        run.slabAxis, run.slabCenter, run.slabWidth, hyb.bandD0);
}

}  // extern "C"
