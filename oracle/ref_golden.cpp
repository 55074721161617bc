// ref_golden.cpp -- drives the reference's own header-only code on given
// inputs to produce golden vectors that pin the oracle.  Compiled against the
// AERO-F sources (-I<reference tree> -DTEMPLATE_FIX) by oracle/Makefile into
// oracle/_ref/ref_golden; nothing from the reference is copied here.
//
// Exercised reference code:
//   RecFcnVanAlbada<5>::compute   (RecFcnDesc.h:703-713 -> RecFcn.h:268-281,432-446)
//   RecFcnLinear<5>::compute      (RecFcnDesc.h, RecFcn.h:240-249)
//   VarFcnSGEuler::conservativeToPrimitive / primitiveToConservative
//                                 (VarFcnSGEuler.h:307-327, 383-394)
//   VarFcnBase::postMultiplyBydVdU / postMultiplyBydUdV
//                                 (VarFcnBase.h:350-400 via VarFcnSGEuler.h:588-620)
//   VarFcnSGEuler::checkReconstructedValues (VarFcnSGEuler.h:90-110)
//   invertDenseMatrix<double,5>   (DenseMatrixOps.h:1006-1185, LINPACK dgefa/dgedi)
//
// Protocol: reads "<kind> <count>" then count records of doubles from
// stdin, writes one line of %.17g outputs per record to stdout.
#include <cstdio>
#include <cstring>
#include <Vector.h>
#include <IoData.h>
#include <RecFcnDesc.h>
#include <VarFcnSGEuler.h>
#include <DenseMatrixOps.h>

// The reference defines these constructors in its parser unit (IoDataCore.C),
// which needs flex/bison/MPI and cannot be built here; the harness only needs
// objects it then fills in field by field.
GasModelData::GasModelData() {}
JWLModelData::JWLModelData() {}
LiquidModelData::LiquidModelData() {}
FluidModelData::FluidModelData() {}

static void put(const double* x, int n) {
  for (int k = 0; k < n; ++k) std::printf(k ? " %.17g" : "%.17g", x[k]);
  std::printf("\n");
}
static bool get(double* x, int n) {
  for (int k = 0; k < n; ++k)
    if (std::scanf("%lf", &x[k]) != 1) return false;
  return true;
}

int main() {
  FluidModelData fm;
  fm.fluid = FluidModelData::PERFECT_GAS;
  fm.rhomin = -1e9; fm.pmin = -1e9;
  fm.gasModel.type = GasModelData::IDEAL;
  fm.gasModel.specificHeatRatio = 1.4;
  fm.gasModel.pressureConstant = 0.0;
  VarFcnSGEuler vf(fm);
  char kind[64];
  int count;
  while (std::scanf("%63s %d", kind, &count) == 2) {
    for (int r = 0; r < count; ++r) {
      if (!std::strcmp(kind, "vanalbada") || !std::strcmp(kind, "linear")) {
        double in[21], a[5], b[5], out[10];
        if (!get(in, 21)) return 1;   // beta, Vi[5], ddVij[5], Vj[5], ddVji[5]
        if (!std::strcmp(kind, "vanalbada")) {
          RecFcnVanAlbada<5> rf(in[0], 0.1);
          rf.compute(in + 1, in + 6, in + 11, in + 16, a, b);
        } else {
          RecFcnLinear<5> rf(in[0], 0.1);
          rf.compute(in + 1, in + 6, in + 11, in + 16, a, b);
        }
        std::memcpy(out, a, sizeof a); std::memcpy(out + 5, b, sizeof b);
        put(out, 10);
      } else if (!std::strcmp(kind, "cons2prim")) {
        double U[5], V[5];
        if (!get(U, 5)) return 1;
        vf.conservativeToPrimitive(U, V);
        put(V, 5);
      } else if (!std::strcmp(kind, "prim2cons")) {
        double V[5], U[5];
        if (!get(V, 5)) return 1;
        vf.primitiveToConservative(V, U);
        put(U, 5);
      } else if (!std::strcmp(kind, "dVdU") || !std::strcmp(kind, "dUdV")) {
        double in[30], out[25];
        if (!get(in, 30)) return 1;   // V[5], mat[25]
        if (!std::strcmp(kind, "dVdU")) vf.postMultiplyBydVdU(in, in + 5, out);
        else vf.postMultiplyBydUdV(in, in + 5, out);
        put(out, 25);
      } else if (!std::strcmp(kind, "check")) {
        double V[5];
        if (!get(V, 5)) return 1;
        double bad = vf.checkReconstructedValues(V, 1, 2, 0, 0, 1) ? 1.0 : 0.0;
        put(&bad, 1);
      } else if (!std::strcmp(kind, "invert5")) {
        double a[25];
        if (!get(a, 25)) return 1;
        int ierr = invertDenseMatrix<double, 5>(a);
        double out[26];
        out[0] = ierr;
        std::memcpy(out + 1, a, sizeof a);
        put(out, 26);
      } else {
        return 2;
      }
    }
  }
  return 0;
}
