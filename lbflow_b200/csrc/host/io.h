// File formats of the LBFlow command line: uint8 geometry, VTI fields and the
// population checkpoint with its sidecar.
//
// The byte layouts are LBFlow's, so its Python tools read our output and we
// read its checkpoints:
//  - geometry: nx*ny*nz raw uint8 labels, x fastest (fileraw.h:231-291);
//  - VTI: VTK ImageData XML header + appended raw FP64 blocks, each preceded
//    by a UInt64 byte count; scalars in name order, then the vector with its
//    components interleaved x, y(, z) (filevti.cpp:39-172);
//  - checkpoint outPath.<t, 10 digits>.rst: raw FP64 post-collision
//    populations [phase][q][voxel] (scsp.cpp:290-302, colorfluid.cpp:789-812);
//  - sidecar .rst.meta (simulator.cpp:345-359) and its load-time checks
//    (simulator.cpp:361-384).
#ifndef LBF_HOST_IO_H
#define LBF_HOST_IO_H

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace lbfhost {

std::vector<uint8_t> loadGeometry(const std::string& path, std::size_t n);

// A VTI file from one dense block laid out as its appended arrays: every
// scalar [N] in order, then the vector [N][components] interleaved.
// sz: reference order sizes ({y,x} or {z,y,x}).
void writeVtiBlocks(const std::string& path, const std::vector<std::size_t>& sz,
                    const std::vector<std::string>& scalars, const std::string& vector, int components,
                    const double* data);

std::string stepName(const std::string& outPath, std::size_t t, const char* ext);

void writeCheckpoint(const std::string& path, const double* f, std::size_t count);
void writeCheckpointMeta(const std::string& path, std::size_t t, std::size_t phases, std::size_t D,
                         std::size_t Q, const std::vector<std::size_t>& sz);
// Throws the reference's messages on a missing/incompatible sidecar or a
// population file of the wrong length.
void validateCheckpoint(const std::string& path, std::size_t t, std::size_t phases, std::size_t D,
                        std::size_t Q, const std::vector<std::size_t>& sz);
std::vector<double> readCheckpoint(const std::string& path, std::size_t count);

}  // namespace lbfhost

#endif
