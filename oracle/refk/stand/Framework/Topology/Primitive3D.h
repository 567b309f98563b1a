#pragma once
// Stand-in for the reference's mesh-geometry header Framework/Topology/Primitive3D.h.
//
// TEST INFRASTRUCTURE ONLY: part of the golden-fixture driver under oracle/.
//
// The reference header declares defaults of the form `Bool& bInside = Bool(false)`
// (Primitive3D.h:142-146), a non-const reference bound to a temporary, which EDG
// and gcc reject. GridHash.h includes it only for the triangle-mesh variant of
// the grid hash and the neighbour query. This stand-in declares just the names
// those mesh kernels use, so their translation units compile; the golden driver
// never launches a mesh kernel, and no particle kernel touches these types.
#include "Core/Vector.h"
#include "Core/Matrix.h"
namespace PhysIKA {
typedef Vector3f Coord3D;
struct Triangle3D {
    Coord3D v[3];
    COMM_FUNC Triangle3D() {}
    COMM_FUNC Triangle3D(const Coord3D& a, const Coord3D& b, const Coord3D& c) { v[0] = a; v[1] = b; v[2] = c; }
};
struct Point3D {
    Coord3D origin;
    COMM_FUNC Point3D() {}
    COMM_FUNC explicit Point3D(const Coord3D& p) : origin(p) {}
    COMM_FUNC float distance(const Triangle3D&) const { return 0.0f; }
};
struct AlignedBox3D {
    Coord3D v0, v1;
    COMM_FUNC AlignedBox3D() {}
    COMM_FUNC AlignedBox3D(const Coord3D& a, const Coord3D& b) : v0(a), v1(b) {}
    COMM_FUNC bool meshInsert(const Triangle3D&) const { return false; }
};
}
