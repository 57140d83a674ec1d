// Instantiation of the solver for the generated model plugin "sme2d_l1".
#include "model_prelude.h"
namespace sme2d_l1 {
#include "sme2d_l1/Model.H"
#include "sme2d_l1/Numerics.H"
}
#include "solver.cuh"
ZSME_DEFINE_MODEL(sme2d_l1)
