// TEST INFRASTRUCTURE ONLY (golden-fixture driver).
//
// The reference translation units the driver compiles also instantiate their
// module classes (DensityPBD<DataType3f>, NeighborQuery<DataType3f>, ...),
// whose host methods and vtables name Framework functions defined in sources
// the driver does not build (Module.cpp, Field.cpp, SceneGraph.cpp, ...). The
// driver never constructs a module. The one Framework function that runs is
// Register(), called by each class's static ClassInfo at start-up; it is given
// a body here that records nothing. Every other such symbol is bound by the
// generated linker script to refk_unreached(), which stops the process if it
// is ever called.
#include <cstdio>
#include <cstdlib>

namespace PhysIKA {
class ClassInfo;
bool Register(ClassInfo*) { return true; }
}  // namespace PhysIKA

extern "C" void refk_unreached(void)
{
    std::fprintf(stderr, "pkref_driver: a Framework function the driver does not provide was called\n");
    std::abort();
}
