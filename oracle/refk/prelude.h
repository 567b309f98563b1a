// Compile environment for the reference's own hot-path translation units.
//
// TEST INFRASTRUCTURE ONLY: part of the golden-fixture driver under oracle/.
//
// The reference's Framework/Framework/FieldVar.h:136 iterates with MSVC's
// `for each (auto fs in sinks)`, which neither EDG nor gcc accept. Every
// Framework header reaches FieldVar.h, so every hot-path translation unit stops
// there. This prelude includes everything FieldVar.h depends on first, then
// FieldVar.h itself with two macros that spell that one statement as the C++11
// `for (auto fs : sinks)` and exist only while that header is parsed; its
// `#pragma once` keeps it from being parsed again later. Field.h:89 uses
// FLT_MAX without <cfloat>, so <cfloat> comes first. No reference file is
// edited or copied.
#pragma once
#include <cfloat>
#include <iostream>
#include <functional>
#include <memory>
#include <string>
#include <vector>
#include "Core/Typedef.h"
#include "Framework/Framework/Field.h"
#include "Framework/Framework/Base.h"
#include "Framework/Framework/Log.h"
#include "Core/Array/MemoryManager.h"
#define each
#define in :
#include "Framework/Framework/FieldVar.h"
#undef in
#undef each
