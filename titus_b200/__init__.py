"""titus_b200: B200-native (sm_100a) CSD energy step of TITUS behind its Settings/SolverCSD/Solve* API."""
from .settings import Settings, Settings3D  # noqa: F401
from .solver import (DoseAdjoint, PencilBeamBatch, SolveBatchedPencilBeams, SolverCSD, SolverCSD3D,  # noqa: F401
                     SolveFirstCollisionSource,
                     SolveFirstCollisionSourceDLR, SolveFirstCollisionSourceDLRHighOrder,
                     SolveFirstCollisionSourceDLRBUGRejection, SolveFirstCollisionSourceDLRParallel,
                     SolveFirstCollisionSourceDLRParallelRejection, scalar_flux)
from .spots import partition, plan_adjoint, plan_dose, plan_objective  # noqa: F401
from .output import write_dlm, write_dose_vtk, write_dose_vtk_3d, write_vtr  # noqa: F401
