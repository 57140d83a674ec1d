// Instantiation of the solver for the generated model plugin "sme1d_l0_malpasset".
#include "model_prelude.h"
namespace sme1d_l0_malpasset {
#include "sme1d_l0_malpasset/Model.H"
#include "sme1d_l0_malpasset/Numerics.H"
}
#include "solver.cuh"
ZSME_DEFINE_MODEL(sme1d_l0_malpasset)
