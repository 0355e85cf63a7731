// Scene ingestion of the CLI drop-in (host code): the Mitsuba XML subset of
// src/mitsuba.rs:137-595 with OBJ meshes (src/obj_loader.rs:11-109) and
// Radiance env maps, and the built-in default scene of src/scene.rs:26-95.
// The result owns every array a tpt_scene_desc points at.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/tinypt_cuda.h"

namespace tpt {

struct LoadedMesh {
    std::vector<double> pos;     // n_vertices * 3
    std::vector<int32_t> idx;    // n_tris * 3
    std::vector<int32_t> mat;    // n_tris
};

struct LoadedScene {
    std::vector<tpt_material> mats;
    std::vector<tpt_sphere> spheres;
    std::vector<LoadedMesh> meshes;
    std::vector<tpt_mesh_desc> mesh_descs;
    std::vector<tpt_instance_desc> instances;
    std::vector<double> env_pixels;
    std::vector<std::string> warnings;
    tpt_scene_desc desc{};
    void finalize();             // points desc at the arrays
};

// Loads a Mitsuba XML scene; film / sampler / integrator values override
// the config's width, height, spp, max_bounces and rr_start
// (src/mitsuba.rs:145-170).  Throws std::runtime_error on a malformed file.
std::unique_ptr<LoadedScene> load_mitsuba(const std::string& path, tpt_render_config& config);

// The built-in scene (src/scene.rs:26-95); env_path (may be empty) is a
// Radiance .hdr env map, else the procedural sky.
std::unique_ptr<LoadedScene> default_scene(const tpt_render_config& config, const std::string& env_path);

// OBJ positions and fan-triangulated faces (src/obj_loader.rs:11-47).
void load_obj(const std::string& path, std::vector<double>& pos, std::vector<int32_t>& idx);

}  // namespace tpt
