"""tomotopy_b200 -- tomotopy's LDA collapsed-Gibbs path on NVIDIA B200 (sm_100a)."""
__version__ = "0.1.0"

from ._lib import lib as _native, TmtError  # noqa: F401,E402  (loads the CUDA library or raises)
from .engine import Engine, Server, synth_corpus, prepare_ids  # noqa: F401,E402
from .models import LDAModel, Document, TermWeight, ParallelScheme, isa  # noqa: F401,E402
