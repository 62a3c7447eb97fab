// Minimal stand-in for Cantera's umbrella header, enough for the reference's
// single-component translation units to compile: they only name the Solution type in
// a shared declaration (src/headers/cantera.hpp:6) and never call into Cantera.
#pragma once
#include <memory>
#include <vector>
namespace Cantera { class Solution; }
