// Host definition of cfd::arrhenius, which the reference declares __host__ __device__
// (src/FiniteRateChem.cuh:28) but defines only in device code (src/FiniteRateChem.cu:1556):
// k = A T^b exp(-Ea/T).  TEST INFRASTRUCTURE ONLY (links the reference's host chemistry).
#include <cmath>
namespace cfd {
double arrhenius(double t, double A, double b, double Ea) { return A * std::pow(t, b) * std::exp(-Ea / t); }
}
