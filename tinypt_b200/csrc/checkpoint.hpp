// Checkpoint files compatible with the reference's HYPCKPT v1 format and
// the film's tile order (host code).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tpt {

struct TileRect { int x0, y0, x1, y1; };

// Tiles of the film in task-id order (src/render.rs:75-100).
std::vector<TileRect> film_tiles(int w, int h, int tile, bool morton);

void save_checkpoint(const std::string& path, uint64_t scene_hash, int w, int h, uint64_t next_id,
                     const double* acc, const double* acc_w);
// false when there is no file or it does not match (magic, version, scene
// hash, size) -- src/checkpoint.rs:86-138 returns None then; throws when
// the file cannot be read or ends early (the reference's io::Error).
bool load_checkpoint(const std::string& path, uint64_t scene_hash, int w, int h, uint64_t& next_id, double* acc,
                     double* acc_w);

// acc += acc_new over the tiles first, first + 1, ... (the tiles a resumed
// render still has to merge).
void merge_tiles(const std::vector<TileRect>& tiles, size_t first, int w, const double* acc_new,
                 const double* w_new, double* acc, double* acc_w);

}  // namespace tpt
