// ParticleIO.cpp -- ParticleWriter frames, the OBJ point reader and the
// lattice fills of ParticleSystem::loadParticles (see ParticleIO.h), plus C
// entry points for hosts and tests that do not link C++.
#include "ParticleIO.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <fstream>
#include <sstream>
#include <stdexcept>

#include "ParticleModules.h"

namespace PhysIKA {

bool writeParticleFrame(const std::string& filename, const Vector3f* pos, const float* color, int n)
{
    // ParticleWriter.cpp:50-80: count, then (x, y, z, color) per particle
    std::ofstream out(filename.c_str(), std::ios::out | std::ios::binary);
    if (!out) return false;
    const int32_t total = n < 0 ? 0 : n;
    out.write(reinterpret_cast<const char*>(&total), sizeof(total));
    std::vector<float> rec((size_t)total * 4);
    for (int i = 0; i < total; ++i) {
        rec[4 * (size_t)i] = pos[i][0];
        rec[4 * (size_t)i + 1] = pos[i][1];
        rec[4 * (size_t)i + 2] = pos[i][2];
        rec[4 * (size_t)i + 3] = color[i];
    }
    if (total > 0) out.write(reinterpret_cast<const char*>(rec.data()), (std::streamsize)(rec.size() * sizeof(float)));
    return (bool)out;
}

bool readParticleFrame(const std::string& filename, std::vector<Vector3f>& pos, std::vector<float>& color)
{
    std::ifstream in(filename.c_str(), std::ios::in | std::ios::binary);
    if (!in) return false;
    int32_t total = 0;
    if (!in.read(reinterpret_cast<char*>(&total), sizeof(total)) || total < 0) return false;
    std::vector<float> rec((size_t)total * 4);
    if (total > 0 && !in.read(reinterpret_cast<char*>(rec.data()), (std::streamsize)(rec.size() * sizeof(float))))
        return false;
    pos.resize((size_t)total);
    color.resize((size_t)total);
    for (int i = 0; i < total; ++i) {
        pos[(size_t)i] = Vector3f(rec[4 * (size_t)i], rec[4 * (size_t)i + 1], rec[4 * (size_t)i + 2]);
        color[(size_t)i] = rec[4 * (size_t)i + 3];
    }
    return true;
}

bool loadObjPoints(const std::string& filename, std::vector<Vector3f>& points, std::vector<Vector3f>& normals)
{
    points.clear();
    normals.clear();
    if (filename.size() < 5 || filename.substr(filename.size() - 4) != std::string(".obj")) {
        Log::sendMessage(Log::Error, "Expected OBJ file with filename of the form <name>.obj");
        return false;
    }
    std::ifstream infile(filename);
    if (!infile) {
        Log::sendMessage(Log::Error, "Failed to open " + filename);
        return false;
    }
    std::string line;
    while (std::getline(infile, line)) {
        const bool is_vn = line.compare(0, 2, "vn") == 0;
        if (line.compare(0, 1, "v") == 0 && !is_vn) {
            std::stringstream data(line);
            char c;
            Vector3f p;
            data >> c >> p[0] >> p[1] >> p[2];
            points.push_back(p);
        } else if (is_vn) {
            std::stringstream data(line);
            char c;
            Vector3f q;
            data >> c >> q[0] >> q[1] >> q[2];
            normals.push_back(q);
        }
    }
    if (normals.size() < points.size()) {
        Log::sendMessage(Log::Warning, "The normal size is not equal to the vertex size!");
        normals.resize(points.size(), Vector3f(0.0f));
    }
    return true;
}

std::vector<Vector3f> latticeBox(Vector3f lo, Vector3f hi, float distance)
{
    std::vector<Vector3f> v;
    if (!(distance > 0.0f)) return v;
    for (float x = lo[0]; x <= hi[0]; x += distance)
        for (float y = lo[1]; y <= hi[1]; y += distance)
            for (float z = lo[2]; z <= hi[2]; z += distance) v.push_back(Vector3f(x, y, z));
    return v;
}

std::vector<Vector3f> latticeBall(Vector3f center, float r, float distance)
{
    std::vector<Vector3f> v;
    if (!(distance > 0.0f)) return v;
    const Vector3f lo(center[0] - r, center[1] - r, center[2] - r);
    const Vector3f hi(center[0] + r, center[1] + r, center[2] + r);
    for (float x = lo[0]; x <= hi[0]; x += distance)
        for (float y = lo[1]; y <= hi[1]; y += distance)
            for (float z = lo[2]; z <= hi[2]; z += distance) {
                // (p - center).norm(): sqrt of x*x + y*y + z*z summed in that order
                const float dx = x - center[0], dy = y - center[1], dz = z - center[2];
                if (std::sqrt(dx * dx + dy * dy + dz * dz) < r) v.push_back(Vector3f(x, y, z));
            }
    return v;
}

template <typename TDataType>
bool ParticleWriter<TDataType>::execute()
{
    const int n = (int)m_position.getElementCount();
    if ((int)m_color_mapping.getElementCount() != n) {
        Log::sendMessage(Log::Error, "ParticleWriter: position and color mapping sizes differ");
        return false;
    }
    std::vector<Coord> pos((size_t)n);
    std::vector<Real> color((size_t)n);
    if (n > 0) {
        if (cudaMemcpy(pos.data(), m_position.getValue().getDataPtr(), sizeof(Coord) * (size_t)n,
                       cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(color.data(), m_color_mapping.getValue().getDataPtr(), sizeof(Real) * (size_t)n,
                       cudaMemcpyDeviceToHost) != cudaSuccess) {
            Log::sendMessage(Log::Error, "ParticleWriter: device copy failed");
            return false;
        }
    }
    const std::string filename = m_output_path + m_name_prefix + std::to_string(m_output_index) + ".txt";
    if (!writeParticleFrame(filename, pos.data(), color.data(), n)) {
        Log::sendMessage(Log::Error, "ParticleWriter: cannot write " + filename);
        return false;
    }
    ++m_output_index;
    return true;
}

// ParticleSystem::loadParticles (ParticleSystem.cpp:34-97): the points become
// the particles (velocities zero).
template <typename TDataType>
void ParticleSystem<TDataType>::loadParticles(std::string filename)
{
    std::vector<Coord> pts, nrm;
    if (!loadObjPoints(filename, pts, nrm)) throw std::runtime_error("loadParticles: cannot read " + filename);
    setParticles(pts, std::vector<Coord>(pts.size(), Coord(0.0f)));
}

template <typename TDataType>
void ParticleSystem<TDataType>::loadParticles(Coord center, Real r, Real distance)
{
    const std::vector<Coord> pts = latticeBall(center, r, distance);
    setParticles(pts, std::vector<Coord>(pts.size(), Coord(0.0f)));
}

template <typename TDataType>
void ParticleSystem<TDataType>::loadParticles(Coord lo, Coord hi, Real distance)
{
    const std::vector<Coord> pts = latticeBox(lo, hi, distance);
    setParticles(pts, std::vector<Coord>(pts.size(), Coord(0.0f)));
}

template class ParticleWriter<DataType3f>;
template void ParticleSystem<DataType3f>::loadParticles(std::string);
template void ParticleSystem<DataType3f>::loadParticles(Vector3f, float, float);
template void ParticleSystem<DataType3f>::loadParticles(Vector3f, Vector3f, float);

}  // namespace PhysIKA

using namespace PhysIKA;

namespace {
int copy_out(const std::vector<Vector3f>& v, float* xyz, int capacity)
{
    const int n = (int)v.size();
    if (xyz != nullptr)
        for (int i = 0; i < n && i < capacity; ++i)
            for (int a = 0; a < 3; ++a) xyz[3 * i + a] = v[(size_t)i][a];
    return n;
}
}  // namespace

extern "C" {

// Writes one ParticleWriter frame from host arrays (xyz: 3n floats, color: n
// floats).  0 on success.
__attribute__((visibility("default"))) int pkf_write_frame(const char* filename, const float* xyz,
                                                           const float* color, int n)
{
    if (!filename || n < 0 || (n > 0 && (!xyz || !color))) return -1;
    std::vector<Vector3f> pos((size_t)n);
    for (int i = 0; i < n; ++i) pos[(size_t)i] = Vector3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    return writeParticleFrame(filename, pos.data(), color, n) ? 0 : -1;
}

// Reads a frame: returns its particle count (-1 if unreadable) and fills up to
// `capacity` particles of xyz (3 per particle) and color.
__attribute__((visibility("default"))) int pkf_read_frame(const char* filename, float* xyz, float* color,
                                                          int capacity)
{
    if (!filename) return -1;
    std::vector<Vector3f> pos;
    std::vector<float> col;
    if (!readParticleFrame(filename, pos, col)) return -1;
    if (color != nullptr)
        for (int i = 0; i < (int)col.size() && i < capacity; ++i) color[i] = col[(size_t)i];
    return copy_out(pos, xyz, capacity);
}

// PointSet::loadObjFile: returns the vertex count (-1 if the file is refused)
// and fills up to `capacity` points and normals (either may be NULL).
__attribute__((visibility("default"))) int pkf_load_obj_points(const char* filename, float* xyz, float* normals,
                                                               int capacity)
{
    if (!filename) return -1;
    std::vector<Vector3f> pts, nrm;
    if (!loadObjPoints(filename, pts, nrm)) return -1;
    copy_out(nrm, normals, capacity);
    return copy_out(pts, xyz, capacity);
}

// ParticleSystem::loadParticles(lo, hi, distance): the point count, up to
// `capacity` points written.
__attribute__((visibility("default"))) int pkf_lattice_box(const float lo[3], const float hi[3], float distance,
                                                           float* xyz, int capacity)
{
    return copy_out(latticeBox(Vector3f(lo[0], lo[1], lo[2]), Vector3f(hi[0], hi[1], hi[2]), distance), xyz,
                    capacity);
}

// ParticleSystem::loadParticles(center, r, distance).
__attribute__((visibility("default"))) int pkf_lattice_ball(const float center[3], float r, float distance,
                                                            float* xyz, int capacity)
{
    return copy_out(latticeBall(Vector3f(center[0], center[1], center[2]), r, distance), xyz, capacity);
}

}  // extern "C"
