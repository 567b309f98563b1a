// ParticleIO.h -- the particle inputs and outputs around the hot path:
//   * ParticleWriter (Dynamics/ParticleSystem/ParticleWriter.h:10-40,
//     ParticleWriter.cpp:44-88): one binary frame per execute(),
//   * PointSet::loadObjFile (Framework/Topology/PointSet.cu:30-86): the
//     vertices ("v") and normals ("vn") of an OBJ file as particles,
//   * ParticleSystem::loadParticles (ParticleSystem.cpp:34-97): lattice fills
//     of a box and of a ball.
// Host code only: frames are copied from device arrays before writing.
#pragma once
#include <string>
#include <vector>

#include "Node.h"

namespace PhysIKA {

// ModuleIO.h:7-19.
class IOModule : public Module {
public:
    std::string getModuleType() override { return "IOModule"; }
};

// A ParticleWriter frame: int32 particle count, then one record of four
// 32-bit floats (x, y, z, color mapping) per particle, native byte order.
bool writeParticleFrame(const std::string& filename, const Vector3f* pos, const float* color, int n);
// Reads a frame written by writeParticleFrame; false on a short or missing file.
bool readParticleFrame(const std::string& filename, std::vector<Vector3f>& pos, std::vector<float>& color);

// PointSet::loadObjFile without the process exit: false (and a Log error) for
// a name not ending in ".obj" or a file that does not open.  Lines beginning
// with 'v' but not "vn" are read as "v x y z" with stream extraction (so a
// "vt" line yields a point whose failed fields are 0, as in the reference);
// "vn" lines are normals, read the same way (one character skipped, so the
// extraction stops at 'n' and the normal is 0, as in the reference); normals
// are padded with zeros up to the vertex count.
bool loadObjPoints(const std::string& filename, std::vector<Vector3f>& points, std::vector<Vector3f>& normals);

// loadParticles(lo, hi, distance): x, y, z stepped by repeated float addition
// from lo while <= hi (x outermost).
std::vector<Vector3f> latticeBox(Vector3f lo, Vector3f hi, float distance);
// loadParticles(center, r, distance): the box [center - r, center + r] filled
// the same way, keeping the points with |p - center| < r.
std::vector<Vector3f> latticeBall(Vector3f center, float r, float distance);

// ParticleWriter: each execute() writes m_position and m_color_mapping (same
// element count) as frame <output path><name prefix><index>.txt and advances
// the index.  The reference writes to a fixed directory with the prefix
// "test_"; here the prefix is settable and defaults to "test_".
template <typename TDataType>
class ParticleWriter : public IOModule {
public:
    typedef typename TDataType::Real Real;
    typedef typename TDataType::Coord Coord;

    void setNamePrefix(std::string prefix) { m_name_prefix = std::move(prefix); }
    void setOutputPath(std::string path) { m_output_path = std::move(path); }
    bool execute() override;
    int getOutputIndex() const { return m_output_index; }

    DeviceArrayField<Coord> m_position{0, "position", "Storing the particle positions!", FieldType::In, nullptr};
    DeviceArrayField<Real> m_color_mapping{0, "ColorMapping", "Storing the particle properties!", FieldType::In,
                                           nullptr};

private:
    int m_output_index = 0;
    std::string m_output_path;
    std::string m_name_prefix = "test_";
};

}  // namespace PhysIKA
