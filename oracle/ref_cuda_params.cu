// Run-time model and shape constants for the reference CUDA propagator —
// TEST INFRASTRUCTURE, linked in place of the reference's src/parameters.cu.
//
// The reference fixes its problem at compile time in src/parameters.cu:11-31
// (`Param::N`, `Param::KMax`, `Param::JMax`, `Param::Step`, bath constants).
// Every other translation unit reads these through the `extern` declarations
// of src/parameters.h, so defining them here from environment variables lets
// one build of the reference run any shape:
//
//   HX_REF_DIM    Hilbert dimension N (default 1024; a power of two, a multiple
//                 of 32 for correct results: the reference's in-place
//                 transpose does nothing otherwise, src/matrix_util.cu:69-80)
//   HX_REF_KMAX   Pade poles; modes = KMAX + 1 (default 2)
//   HX_REF_JMAX   exclusive hierarchy depth bound (default 3)
//   HX_REF_DT     time step (default 0.1)
//   HX_REF_BETA   inverse temperature Betah (default 3)
//   HX_REF_ZETA   coupling strength Zeta (default 0.01)
//
// The remaining values are the reference's compiled model constants
// (src/parameters.cu:11-31), unchanged.
#include "parameters.h"

#include <cmath>
#include <cstdlib>
#include <string>

namespace {

int env_int(const char* name, int fallback)
{
    const char* v = std::getenv(name);
    return (v && *v) ? std::atoi(v) : fallback;
}

double env_double(const char* name, double fallback)
{
    const char* v = std::getenv(name);
    return (v && *v) ? std::atof(v) : fallback;
}

}  // namespace

const double Param::PI = 4.0 * std::atan(1.0);
const Complex iConst = make_Complex(0, 1.0);

const int Param::N = env_int("HX_REF_DIM", 1 << 10);
const int Param::N2 = Param::N * Param::N;
const double Param::Delta = 0;
const double Param::Omega0 = 1.0;
const double Param::Dlong = 1.0;
const double Param::Dtrans = 1.0;
const double Param::JNaver = 0.6;
const bool Param::IsSquare = false;

double Param::Step = env_double("HX_REF_DT", 0.1);
int Param::IntegrationNum = 4;

double Param::Betah = env_double("HX_REF_BETA", 3.0);
const double Param::Gamma = 1;
double Param::Zeta = env_double("HX_REF_ZETA", 0.01);

const int Param::KMax = env_int("HX_REF_KMAX", 2);
const int Param::JMax = env_int("HX_REF_JMAX", 3);

const bool Param::FromBoltzman = true;
const int Param::OutputNum = 1;
const int Param::SnapShotNum = -1;
std::string Param::Filename = "";

cublasHandle_t cublasHandle;
