"""B200 implementation of CompactLES.jl's RHS-and-step hot path.

Host-side mirror of the reference's operator interface (plan_direction /
apply_along!, Solver / compute_rhs! / step! / max_rate / filter_state! /
run!) over the C ABI of libcles.so (include/cles.h).  The CUDA library is
required: every compute call goes through it and raises if it is missing.
"""
from . import abi
from .problem import (ArtParams, AxisBC, CartesianMetric, ConstantBodyForce, CylindricalMetric, DirichletBC,
                      ExtrapolationBC,
                      IdealMixture, IdealSpecies, NoSlipWallBC, NSCBCInflowBC, NSCBCOutflowBC, Numerics, OriginBC,
                      PER3, PeriodicBC, PoleBC, Prim, Problem, SlipWallBC, SphericalMetric, StepControl, Stretch,
                      SwitchableBC, Transport, sine_cluster,
                      conserved_from_prim, coords, grid_spacing, initialize, interior_slices,
                      problem_desc, single_species, solver_desc, state_shape, tanh_blend,
                      taylor_green_problem)
from .api import (ClesError, Context, DirPlan, Solver, SolverFailure, apply_along, build, check_step,
                  compact_filter, default_context, grid, kernel_launches, lele_d1_10, lele_d1_6, lib,
                  pade_d1_4, plan_direction, profile_enable, profile_read, setup, Server, Batch)
from . import scenarios
from .split import LineExchange, SplitPlan, exchange_halos, split_apply_along
from .nasa9 import Nasa9Interval, Nasa9Mixture, Nasa9Species, nasa9_constant_cp, read_nasa9
from .decomp import Decomp, LocalGroup, TorchExchange, assemble, local_range
