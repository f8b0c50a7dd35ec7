"""B200 docking engine: host package over the CUDA C ABI (libudock_b200.so)."""
from .model import Box, Ligand, Receptor, parse_ligand, parse_ligands, parse_receptor  # noqa: F401
from .engine import (Engine, EngineError, DockParams, DockResult, MODE_DIRECT, MODE_GRID,  # noqa: F401
                     GRID_F16, GRID_F32, load_library, make_record, split_record, record_len)
