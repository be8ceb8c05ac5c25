"""lmb200 -- the LatticeMatrices.jl Dirac-operator / D'D-CG path on B200.

Host-side mirror of the reference's operator API over liblmb200.so (C ABI in
include/lmb200.h).  Julia names map as `mul!` -> `mul_`, `cg!` -> `cg_`,
`solve!` -> `solve_`, `update_clover!` -> `update_clover_`, `D'` ->
`adjoint(D)`.
"""
from ._lib import ArgumentError, DimensionMismatch, LMBError, load, EXPORTED, LIB_PATH  # noqa: F401
from .lattice import (LatticeMatrix, clear_matrix_, ensure_halo_,  # noqa: F401
                      halo_is_dirty, mark_halo_dirty_, set_halo_, similar,
                      substitute_)
from .operators import (CloverFieldStrength4D, WilsonDiracCloverOperator4D,  # noqa: F401
                        WilsonDiracOperator4D, adjoint, mul_,
                        StaggeredDiracOperator4D, HISQLinks4D,
                        HISQDiracOperator4D,
                        mul_cached_clover_, mul_cached_clover_adjoint_,
                        update_clover_)
from .hisq import (HISQDiracCache4D, hisq_fat7_level1_,  # noqa: F401
                   hisq_fermion_force_, hisq_link_pullback_,
                   hisq_fat7_level2_, hisq_links_from_thin, hisq_naik_links_,
                   hisq_project_u3_, mul_cached_hisq_,
                   mul_cached_hisq_adjoint_)
from .clover import wilson_clover_fermion_force_, wilson_clover_link_pullback_  # noqa: F401
from .domainwall import (D5DW_GeneralizedDomainwallOperator5D,  # noqa: F401
                         D5DW_MobiusDomainwallOperator5D)
from .inputs import gaussian_fermion, random_su3_links  # noqa: F401
from .solver import (CGResult, DdagDOp, cg_, cg_batched_, dot,  # noqa: F401
                     operator_timing, pseudofermion_action, solve_, solve_evenodd_)
