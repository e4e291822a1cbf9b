"""B200-native density-and-potential stage of the PGalF galaxy finder.

The CUDA kernels and the C ABI live in ``libgf.so`` (sources under ``csrc/``,
declarations in ``include/gf.h``); this package holds the ctypes binding and
the host side around it:

* ``batch``    — the batched device API over torch buffers: ``stage_run`` (the
  whole stage on many halos), ``PipelinedStage`` (halo chunks on their own
  streams and threads), kNN, mesh, potential, core finding;
* ``dropin``   — the reference's entry points with their signatures and
  meaning (``findsphdensity``, ``assign_density_TSC``, ``Self_Halo_Potent``,
  ``finddenpeak``, ...), raising ``GFError`` where the reference exits;
* ``autograd`` — the differentiable mesh and kNN densities;
* ``centres``  — gradient-ascent refinement of galaxy centres;
* ``fofio``    — the FoF catalogue input and GALFIND output formats;
* ``shard``    — halo partition and output gather across ranks;
* ``synth``    — seeded synthetic catalogues;
* ``build`` / ``tune`` — the sm_100a build and its autotuner.
"""
from ._lib import GFError, lib  # noqa: F401
