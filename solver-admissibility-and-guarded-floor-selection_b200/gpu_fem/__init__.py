"""B200-native guarded SIMP-floor linear-elasticity solve.

Module and class names mirror the reference package ``gpu_fem`` so its
experiment drivers and callers find the same API:

    gpu_fem.presets.get_preset, gpu_fem.bc_generator.generate_bc,
    gpu_fem.pub_simp_solver.{KE_UNIT_3D, _edof_table_3d, _build_density_filter, StepState},
    gpu_fem.solver_v2.{MatrixFreeKff, NodeBlockJacobiMF, _cupy_pcg},
    gpu_fem.multigrid_v4.{GalerkinMatFreeGMG, _cupy_fgmres},
    gpu_fem.cuda_fused_matvec.FusedMatvec, gpu_fem.paper4._build_components,
    gpu_fem.policy.GuardedFloorPolicy, gpu_fem.solver_v4.SolverV4,
    gpu_fem.simp_gpu.{TO3DParams, run_simp_surrogate_gpu},
    gpu_fem.pub_baseline_controller.ScheduleOnlyController,
    gpu_fem.local_agents.PureFEMRouter.

The compute path is libsimpfem.so (sm_100a CUDA); importing this package does
not touch the GPU.
"""

__all__ = ["presets", "bc_generator", "pub_simp_solver", "solver_v2", "multigrid_v4", "policy", "paper4"]
