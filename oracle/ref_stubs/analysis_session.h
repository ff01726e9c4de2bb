// TEST INFRASTRUCTURE: stands in for the reference's analysis_session.h when its
// data_export.cpp is compiled for the CSV wire-format tests (oracle/build_ref.sh). The real
// header pulls in the GUI (ImGui, plot views); data_export.cpp needs from it only the type
// of the phase-portrait export's argument, which is out of this engine's path and never
// called by the tests. Declared here with the one member that export touches.
#pragma once
#include <vector>

#include "parametric_engine.h"

struct AnalysisResult {
    std::vector<std::vector<std::vector<double>>> trajectories;  // [initial condition][step][coordinate]
};
