"""Simulation configuration (drop-in for the reference's config/settings.py:9-230).

Same dataclasses, field names and defaults as the reference, so existing
driver code and saved ``simulation_config.json`` files keep working.  Two
reference quirks are kept on purpose:
  * ``VanGenuchtenParameters.m`` defaults to 1 - 1/1.56 (evaluated once at
    class definition, settings.py:17); setting ``n`` alone does not change it;
  * ``SimulationConfig.validate`` keeps the reference's whitelist.
Additions (new names only): ``SolverParameters.precision`` ("fp64" or
"mixed"), ``inner_tol``/``refine_maxiter`` for the mixed path, and
``MeshParameters`` accepting ``mesh_dir=None`` to use the structured
generators instead of CSV files.
"""
from dataclasses import asdict, dataclass, field
from pathlib import Path
from typing import Any, Dict, Optional, Tuple

import numpy as np

_N_DEFAULT = 1.56


@dataclass
class VanGenuchtenParameters:
    Ks: float = 0.2496
    thetas: float = 0.43
    thetar: float = 0.078
    alpha: float = 3.6
    n: float = _N_DEFAULT
    m: float = 1 - 1 / _N_DEFAULT

    def to_array(self) -> np.ndarray:
        """[alpha, theta_s, theta_r, n, m, Ks] (van_genuchten.py:24)."""
        return np.array([self.alpha, self.thetas, self.thetar, self.n, self.m, self.Ks], dtype=np.float64)

    def to_dict(self) -> Dict:
        return asdict(self)


@dataclass
class SoluteParameters:
    DL: float = 0.5
    DT: float = 0.1
    Dm: float = 0.0
    c_init: float = 0.1
    c_inlet: float = 1.0

    def to_dict(self) -> Dict:
        return asdict(self)


@dataclass
class ExponentialParameters:
    Ks: float = 0.1
    thetas: float = 0.45
    thetar: float = 0.15
    alpha0: float = 0.164

    def to_array(self) -> np.ndarray:
        """[alpha0, theta_s, theta_r, Ks] (exponential.py:24)."""
        return np.array([self.alpha0, self.thetas, self.thetar, self.Ks], dtype=np.float64)

    def to_dict(self) -> Dict:
        return asdict(self)


@dataclass
class NitrogenParameters:
    DL: float = 0.04
    DT: float = 0.0004
    Dm: float = 0.288e-4
    rho: float = 1.6e-6
    Kd: float = 0.34e-6
    mu1: float = 0.12
    mu2: float = 0.048
    mu3: float = 0.012
    c_init_NH4: float = 0.0
    c_init_NO2: float = 0.0
    c_init_NO3: float = 0.0
    c_inlet_NH4: float = 50.0
    c_inlet_NO2: float = 0.0
    c_inlet_NO3: float = 20.0

    def to_array(self) -> np.ndarray:
        return np.array([self.DL, self.DT, self.Dm, self.rho, self.Kd, self.mu1, self.mu2, self.mu3],
                        dtype=np.float64)

    def to_dict(self) -> Dict:
        return asdict(self)


@dataclass
class TimeSteppingParameters:
    dt_init: float = 1e-5
    Tmax: float = 1.0
    m_it: int = 5
    M_it: int = 7
    W_it: int = 10
    lambda_amp: float = 2.0
    lambda_red: float = 0.5

    def to_dict(self) -> Dict:
        return asdict(self)


@dataclass
class SolverParameters:
    solver_type: str = "gmres"
    precond_type: str = "ilu"
    tol: float = 1e-10
    maxiter: int = 100
    restart: int = 30
    precond_params: Dict[str, Any] = field(default_factory=lambda: {"alpha": 1.0, "omega": 1.0, "block_size": 2})
    precision: str = "fp64"          # addition: "fp64" | "mixed" (FP32 Krylov inside FP64 refinement)
    inner_tol: float = 1e-4          # addition: mixed path, relative tolerance of each FP32 solve
    refine_maxiter: int = 30         # addition: mixed path, refinement cap

    def to_dict(self) -> Dict:
        return asdict(self)


@dataclass
class MeshParameters:
    mesh_size: str = "25"
    mesh_dir: Optional[str] = "data/mesh"
    test_case: str = "Test1"

    @property
    def mesh_files(self) -> Tuple[Path, Path]:
        base = Path(self.mesh_dir if self.mesh_dir is not None else ".")
        if self.test_case == "SoluteTest":
            return base / "solute" / "p_Pinns.csv", base / "solute" / "t_Pinns.csv"
        if self.test_case == "Test3D":
            return base / "richards" / "p_3D.csv", base / "richards" / "t_3D.csv"
        return base / "richards" / f"p{self.mesh_size}.csv", base / "richards" / f"t{self.mesh_size}.csv"

    def validate_mesh_files(self) -> bool:
        p, t = self.mesh_files
        if not p.exists():
            raise FileNotFoundError(f"Points file not found: {p}")
        if not t.exists():
            raise FileNotFoundError(f"Triangles file not found: {t}")
        return True

    def to_dict(self) -> Dict:
        p, t = self.mesh_files
        return {"mesh_size": self.mesh_size, "mesh_dir": None if self.mesh_dir is None else str(self.mesh_dir),
                "test_case": self.test_case, "points_file": str(p), "triangles_file": str(t)}


@dataclass
class SimulationConfig:
    exponential: ExponentialParameters = field(default_factory=ExponentialParameters)
    van_genuchten: VanGenuchtenParameters = field(default_factory=VanGenuchtenParameters)
    solute: SoluteParameters = field(default_factory=SoluteParameters)
    nitrogen: NitrogenParameters = field(default_factory=NitrogenParameters)
    time: TimeSteppingParameters = field(default_factory=TimeSteppingParameters)
    solver: SolverParameters = field(default_factory=SolverParameters)
    test_case: str = "Test1"
    save_frequency: int = 1

    def __post_init__(self):
        self.mesh = MeshParameters(test_case=self.test_case)

    def validate(self) -> bool:
        valid_tests = {"Test1", "Test2", "Test3", "Test3D", "SoluteTest"}
        valid_mesh_sizes = {"25", "50", "100", "4096"}
        valid_solvers = {"gmres", "cg", "bicgstab"}
        if self.test_case not in valid_tests:
            raise ValueError(f"Invalid test case. Must be one of {valid_tests}")
        if self.test_case not in ["SoluteTest", "Test3D"] and self.mesh.mesh_size not in valid_mesh_sizes:
            raise ValueError(f"Invalid mesh size for Richards test. Must be one of {valid_mesh_sizes}")
        if self.solver.solver_type not in valid_solvers:
            raise ValueError(f"Invalid solver type. Must be one of {valid_solvers}")
        self.mesh.validate_mesh_files()
        return True

    def to_dict(self) -> Dict:
        return {"exponential": self.exponential.to_dict(), "van_genuchten": self.van_genuchten.to_dict(),
                "solute": self.solute.to_dict(), "time": self.time.to_dict(), "solver": self.solver.to_dict(),
                "mesh": self.mesh.to_dict(), "test_case": self.test_case, "save_frequency": self.save_frequency}


def create_config_from_dict(config_dict: Dict[str, Any]) -> SimulationConfig:
    return SimulationConfig(
        exponential=ExponentialParameters(**config_dict.get("exponential", {})),
        van_genuchten=VanGenuchtenParameters(**config_dict.get("van_genuchten", {})),
        solute=SoluteParameters(**config_dict.get("solute", {})),
        time=TimeSteppingParameters(**config_dict.get("time", {})),
        solver=SolverParameters(**config_dict.get("solver", {})),
        test_case=config_dict.get("test_case", "Test1"),
        save_frequency=config_dict.get("save_frequency", 1))


default_config = SimulationConfig()
