// Instantiation of the solver for the generated model plugin "sme2d_l2".
#include "model_prelude.h"
namespace sme2d_l2 {
#include "sme2d_l2/Model.H"
#include "sme2d_l2/Numerics.H"
}
#include "solver.cuh"
ZSME_DEFINE_MODEL(sme2d_l2)
