/* pme_direct.h -- C ABI of the B200 direct-space (real-space) PME nonbonded engine.
 *
 * The other half of Ewald beside pme_recip.h: the role of CudaPMEDirectForce<long long, float>
 * (ap-hynninen/gpu_recip CudaPMEDirectForce.h:27-205) together with the topological exclusions of
 * CudaTopExcl (CudaTopExcl.cu:6-80).  Pairs within roff under the minimum image of an orthorhombic
 * box get shifted Lennard-Jones (VDW_VSH) and Ewald real-space electrostatics (EWALD), the models
 * the reference's direct test runs (gpu_direct.cu:151-152); the 1-4 inclusion and exclusion lists
 * get the reference's 1-4 terms.  Forces are gradients (+dE/dx, CHARMM convention) ADDED to an
 * int64 SoA array at 2^40 (Force<long long>); energies "vdw", "elec", "excl" and the virial
 * accumulate until cleared.  Unlike the reference, no neighbour-list object is passed: every
 * calc_force bins the atoms into cells itself.
 *
 * Every call is asynchronous on the handle's stream except pme_direct_get_energy_virial (which
 * synchronises) and the set_* calls that upload tables (which synchronise the stream first).
 * Status codes are those of pme_recip.h.
 */
#ifndef PME_DIRECT_H
#define PME_DIRECT_H

#include "pme_recip.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Models, numbered as CudaDirectForceTypes.h:60-63. */
enum { PME_VDW_NONE = 0, PME_VDW_VSH = 1 };
enum { PME_ELEC_NONE = 0, PME_ELEC_EWALD = 101 };

typedef struct pme_direct pme_direct;

PME_API int pme_direct_create(void* stream, pme_direct** out);                 /* ctor, CudaPMEDirectForce.cu:62-100 */
PME_API int pme_direct_destroy(pme_direct* h);
PME_API int pme_direct_set_stream(pme_direct* h, void* stream);

/* setup(boxx, boxy, boxz, kappa, roff, ron, e14fac, vdw_model, elec_model) (CudaPMEDirectForce.cu:151-215).
 * roff must not exceed half the shortest box edge (minimum image).  ron is accepted and unused
 * by VDW_VSH.  Other models return PME_EUNSUPPORTED. */
PME_API int pme_direct_setup(pme_direct* h, double boxx, double boxy, double boxz, double kappa,
                             double roff, double ron, double e14fac, int vdw_model, int elec_model);
PME_API int pme_direct_set_box_size(pme_direct* h, double boxx, double boxy, double boxz);

/* (c6, c12) pairs of the packed lower triangle of vdW types: pair (a >= b) at index
 * a (a + 1) / 2 + b (CudaDirectForce_util.h:265-278); nvdwparam = 2 * pairs.  As
 * set_vdwparam / set_vdwparam14 (CudaPMEDirectForce.cu:362-510), host floats. */
PME_API int pme_direct_set_vdwparam(pme_direct* h, int nvdwparam, const float* h_vdwparam);
PME_API int pme_direct_set_vdwparam14(pme_direct* h, int nvdwparam, const float* h_vdwparam);
/* vdW type (0-based) of every coordinate, in the coordinates' order (set_vdwtype, host). */
PME_API int pme_direct_set_vdwtype(pme_direct* h, int ncoord, const int* h_vdwtype);

/* Topological exclusions as CHARMM's iblo14 / inb14 (CudaTopExcl(ncoord, iblo14, inb14)): atom i's
 * partners are |inb14[iblo14[i-1] .. iblo14[i]-1]| (1-based), numbered in the system's original
 * order.  loc2glo[i] (0-based) is the original index of coordinate i, or NULL for the identity
 * (the reference passes it to its neighbour-list build).  Excluded pairs, and every atom with
 * itself, are left out of calc_force.  Host arrays. */
PME_API int pme_direct_set_exclusions(pme_direct* h, int ncoord, const int* iblo14, const int* inb14,
                                      const int* loc2glo);

/* 1-4 lists (set_14_list, CudaPMEDirectForce.cu:575-596): (i, j, ishift) triples in the
 * coordinates' order, ishift = 13 + dx + 3 dy + 9 dz for the image of j (gpu_utils.h:312-320).
 * in14 pairs get the 1-4 vdW parameters and (erfc + e14fac - 1) electrostatics, ex14 pairs the
 * exclusion correction -qq erf(kappa r)/r.  Host arrays. */
PME_API int pme_direct_set_14_list(pme_direct* h, int nin14, int nex14, const int* in14, const int* ex14);

/* calc_force(xyzq, nlist, calc_energy, calc_virial, stride, force) (CudaPMEDirectForce.cu:719-780):
 * xyzq device float4[ncoord]; force device int64[3 * stride], stride >= ncoord, added to. */
PME_API int pme_direct_calc_force(pme_direct* h, const void* xyzq, int ncoord, int calc_energy,
                                  int calc_virial, int stride, long long* force);
/* calc_14_force(xyzq, calc_energy, calc_virial, stride, force) (CudaPMEDirectForce.cu:671-717). */
PME_API int pme_direct_calc_14_force(pme_direct* h, const void* xyzq, int calc_energy, int calc_virial,
                                     int stride, long long* force);

PME_API int pme_direct_clear_energy_virial(pme_direct* h);
/* Energies (kcal/mol) and the virial tensor (row-major; the reference's sign, gpu_direct.cu:67-70)
 * accumulated since the last clear.  Synchronises the stream. */
PME_API int pme_direct_get_energy_virial(pme_direct* h, double* energy_vdw, double* energy_elec,
                                         double* energy_excl, double* virial9);

#ifdef __cplusplus
}
#endif

#endif /* PME_DIRECT_H */
