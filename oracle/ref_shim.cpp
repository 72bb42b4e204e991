// Test infrastructure only: link shim for building the reference CPU path as an oracle.
//
// The reference's residual/update path (src/*.cpp of rameshkolluru43/CFD_Solver_withCUDA) links
// against 13 symbols that live in files needing jsoncpp / boost / VTK, which are not built here
// (src/Configuration_Read.cpp:10-21,23,126, src/Mesh_Loader.cpp:102, src/Dir_Files.cpp).
// This file provides those symbols so the unmodified reference sources link into
// oracle/_ref/libcfdref.so.  Configuration is set by the harness (ref_harness.cpp) instead of JSON.
#include "definitions.h"
#include "Globals.h"

// src/Configuration_Read.cpp:10 — limiter coefficients (set by the harness).
double Limiter_Zeta = 0.5, Limiter_Zeta1 = 0.5;
// src/Configuration_Read.cpp:14-16 — boundary / initial condition records.
InletCondition inletCond;
ExitCondition exitCond;
InitialCondition initCond;
// src/Configuration_Read.cpp:19,21 — mesh metadata and names.
MeshParams meshParams;
string gridDir, Test_Case_Name = "oracle", Test_Case_JSON_File;

// JSON readers and directory helpers are not on the residual/update path.
void readJSON(const std::string &) {}
void parseTestCaseJSON(const std::string &) {}
bool Load_Mesh(const std::string &) { return false; }
void createOutputDirectories() {}
