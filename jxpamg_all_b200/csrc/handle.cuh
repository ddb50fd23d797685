// The object behind the C handle jxcpr_solver (shared by every file of the ABI).
#pragma once

#include "solver.cuh"

struct jxcpr_solver {
    jxcpr::Solver s;
};
