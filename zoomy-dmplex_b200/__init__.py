"""B200-native shallow-water-moment (SME) time step.

A from-scratch sm_100a implementation of the hot path of ZoomyLab/zoomy-dmplex:
the explicit MUSCL transport update (``TransportStep`` driven by
``MUSCLSolver``) and the implicit per-cell source (``SourceStep``), behind the
reference's generated ``Model<T>``/``Numerics<T>`` plugin interface.

Layers:
  mesh      -- meshes and finite-volume geometry (DMPlex conventions)
  settings  -- the solver subset of the reference's JSON settings
  models/   -- generated model plugins (Model.H / Numerics.H) + generator
  csrc/     -- CUDA kernels and the C ABI (libzsme.so)
  native    -- ctypes binding of the C ABI
  solver    -- MUSCLSolver-shaped host driver over the C ABI
"""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
MODELS_DIR = os.path.join(PKG_DIR, "models")
