"""alpacc_b200: a B200-native (sm_100a) backend for alpacc grammars.

Host side: ``tables`` builds a grammar's lexer and LLP(q,k) tables (the
restated generator), ``api`` runs the CUDA kernels of ``_lib/libalpacc_b200.so``
through the C ABI in ``include/alpacc_b200.h``.
"""

__all__ = ["api", "tables", "synth", "build"]
