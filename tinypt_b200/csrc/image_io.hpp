// Image files of the CLI drop-in (host code): output formats and the
// Radiance reader.
#pragma once

#include <string>
#include <vector>

namespace tpt {

// Writes linear RGB pixels (w*h*3 f64, row 0 at the top) in the format the
// extension selects (src/output.rs:59-132): .exr -> ACEScg float32
// (single part, uncompressed), .hdr -> Radiance RGBE, anything else -> PPM
// (P3) after exposure (2^exposure), tonemap (0 none, 1 ACES fitted) and
// sRGB encoding.  Throws std::runtime_error on failure.
void write_image(const std::string& path, int w, int h, const double* rgb, double exposure, int tonemap);

// Reads a Radiance .hdr file (src/hdr.rs:20-60) into linear RGB, row 0 at
// the top.
void read_hdr(const std::string& path, int& w, int& h, std::vector<double>& rgb);

}  // namespace tpt
