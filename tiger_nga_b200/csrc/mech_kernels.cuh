// Builds the operation table of one generated mechanism.
#pragma once
#include "kernels.cuh"
#include "props_kernels.cuh"

namespace tng {

template <class Mech>
MechOps make_ops(const char* const* species, const double (*wmol)[Mech::NS], int nelem, const char* const* elements,
                 const double* elem, const SvLayout* svl, const double* hd0, const double* hd1, const int* hi,
                 const int* ci, const SolverKernels* sk) {
  MechOps o{};
  o.name = Mech::NAME;
  o.ns = Mech::NS;
  o.nslot = Mech::NSLOT;
  o.nm = Mech::NM;
  o.nelem = nelem;
  o.species = species;
  o.wmol[0] = wmol[0];
  o.wmol[1] = wmol[1];
  o.elements = elements;
  o.elem = elem;
  o.rhs = &launch_rhs<Mech>;
  o.sv_layout = svl;
  o.sv_hd[0] = hd0;
  o.sv_hd[1] = hd1;
  o.sv_hi = hi;
  o.sv_ci = ci;
  o.sk = sk;
  o.props = &launch_props<Mech>;
  return o;
}

}  // namespace tng
