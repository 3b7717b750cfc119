"""Where queries find their inputs and the worker plugin (the reference's
system/tmine/locations.py).  Roots come from the environment, else from the
current directory's inputs/ tree:

  EVX_MOTIF_ROOT  (default ./inputs/motifs)
  EVX_GRAPH_ROOT  (default ./inputs/graphs)
"""
import os

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def inputMotifsRoot() -> str:
    return os.environ.get("EVX_MOTIF_ROOT", os.path.join(os.getcwd(), "inputs", "motifs"))


def inputGraphRoot() -> str:
    return os.environ.get("EVX_GRAPH_ROOT", os.path.join(os.getcwd(), "inputs", "graphs"))


def dynLibPath() -> str:
    """The prebuilt worker plugin (one plugin serves every motif)."""
    return os.path.join(PKG, "libEVX.so")


def randFilePath() -> str:
    """Random-feature file (raw int32; the reference hard-codes its path): node /
    edge predicates and filters read it; queries without them need none."""
    return os.environ.get("EVX_RAND_FILE", "")
