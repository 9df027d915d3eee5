"""The program alpacc's CUDA generator emits, as a stream tool on this backend.

Reads the input from stdin in pieces, lexes each piece on the GPU as it
arrives (the DFA state and token start carried from piece to piece), and
writes one ASCII line ``start end terminal`` per token, the format of
``WriteAscii`` (cuda/lexer.cu:421-426) printed by ``lexer_stream``
(cuda/lexer.cu:452-543) from the generated ``main``
(src/Alpacc/Generator/Cuda/Generator.hs:36-50).  Exits 0 when the input is
accepted and 255 otherwise (that ``main`` returns -1).

One difference, on purpose: ignored tokens are not printed.  The reference's
kernel tests ``IGNORE_TERMINAL`` while its generator defines ``IGNORE_TOKEN``
(cuda/lexer.cu:327-331, src/Alpacc/Generator/Cuda/Lexer.hs:59), so it prints
them; this tool prints what the generated Futhark lexer and alpacc's own
``tokenize`` produce.

    python -m alpacc_b200.lexstream GRAMMAR [--piece BYTES] [--names] < input
"""

from __future__ import annotations

import argparse
import sys

from . import tables
from .api import Grammar


def _lines(term, start, end, names) -> bytes:
    if names is None:
        rows = zip(start.tolist(), end.tolist(), term.tolist())
        return "".join("%d %d %d\n" % r for r in rows).encode()
    return "".join("%d %d %s\n" % (a, b, names[t]) for a, b, t in
                   zip(start.tolist(), end.tolist(), term.tolist())).encode()


def run(grammar: str, src, out, piece: int = 16 << 20, names: bool = False, device: int = 0) -> int:
    """Lex `src` (a binary file object) in `piece`-byte reads, writing lines to
    `out` (a binary file object).  Returns the exit status."""
    g = Grammar(tables.load(grammar, "lexer"), device=device)
    nm = g.tables.terminal_names if names else None
    s = g.lex_stream(piece + 1)
    try:
        first = 0

        def flush(k):
            if k > first:
                m = k - first
                out.write(_lines(s.term[:m].cpu().numpy(), s.start[:m].cpu().numpy(),
                                 s.end_[:m].cpu().numpy(), nm))

        while True:
            buf = src.read(piece)
            if not buf:
                break
            s.window(first)
            s.push(buf)
            k = s.tokens()
            flush(k)
            first = k
        s.window(first)
        _, ok = s.finish()
        flush(s.tokens())  # the last token, also when the input is rejected
        out.flush()
        return 0 if ok else 255
    finally:
        s.close()
        g.close()


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m alpacc_b200.lexstream",
                                 description="lex stdin on the GPU, one 'start end terminal' line per token")
    ap.add_argument("grammar", help="a .alp file or a bundled grammar name (json, sexp, arithmetic, ...)")
    ap.add_argument("--piece", type=int, default=16 << 20, help="bytes read and lexed at a time (default 16 MiB)")
    ap.add_argument("--names", action="store_true", help="print terminal names instead of ids")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.piece <= 0:
        ap.error("--piece must be positive")
    return run(a.grammar, sys.stdin.buffer, sys.stdout.buffer, a.piece, a.names, a.device)


if __name__ == "__main__":
    sys.exit(main())
