"""Grammar front end: the `.alp` file format, its regular expressions, and the
grammar transforms that fix every terminal, symbol and production id.

This is host-side table-generation code (it runs once per grammar, never on the
hot path).  It restates, in Python, the parts of alpacc that decide the integer
ids a generated parser emits:

* `.alp` syntax: ``src/Alpacc/CFG.hs:172-235`` (params, terminal rules,
  nonterminal rules, string-literal terminals) and
  ``src/Alpacc/Lexer/RegularExpression.hs:81-215`` (regex syntax).
* grammar transforms: ``extendByTerminals`` (``src/Alpacc/Grammar.hs:356-378``),
  ``addUnusedTerminal`` (``src/Alpacc/Grammar.hs:347-354``) and
  ``augmentGrammar`` (``src/Alpacc/Grammar.hs:194-215``), composed as in
  ``parsingGrammar`` (``src/Alpacc/Grammar.hs:393-398``).
* id orderings: ``encodeSymbols`` / ``encodeTerminals``
  (``src/Alpacc/Encode.hs:122-162``), lexer terminal priority
  (``src/Alpacc/CFG.hs:159-170``, ``src/Alpacc/Lexer/DFA.hs:326-331``), names
  (``src/Alpacc/Generator/Analyzer.hs:97-104,140-147``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple


class GrammarError(Exception):
    """Raised for grammars alpacc itself rejects (syntax, epsilon tokens,
    nonproductive rules, LL/LLP conflicts)."""


# --------------------------------------------------------------------------
# Terminals and symbols
# --------------------------------------------------------------------------

@dataclass(frozen=True, order=True)
class T:
    """A grammar terminal.  ``lit`` is False for a named terminal (``T name``)
    and True for a string literal (``TLit text``).  Ordering follows Haskell's
    derived ``Ord T`` (``src/Alpacc/Grammar.hs:90``): every named terminal sorts
    before every literal, then by text (code point order)."""

    lit: bool
    name: str

    def pretty(self) -> str:
        return '"%s"' % self.name if self.lit else self.name


@dataclass(frozen=True)
class NT:
    name: str


# A right-hand-side symbol is ('t', T) or ('n', NT).
Sym = Tuple[str, object]


# --------------------------------------------------------------------------
# Regular expressions
# --------------------------------------------------------------------------
# Regex AST (``src/Alpacc/Lexer/RegularExpression.hs:38-45``):
#   ('eps',) | ('lit', bytes) | ('range', (bytes, ...)) | ('star', r)
#   | ('alt', r, r) | ('cat', r, r)

_ESCAPES = {
    "\\": "\\", "/": "/", "[": "[", "]": "]", "(": "(", ")": ")", "*": "*",
    "+": "+", "|": "|", "s": " ", "t": "\t", "n": "\n", "r": "\r", "?": "?",
}
_NOT_PRINT = set("\\/[]()*|+?")


def _is_space(c: str) -> bool:
    return c.isspace()


def _is_print(c: str) -> bool:
    return c.isprintable()


def produces_epsilon(r) -> bool:
    """``producesEpsilon`` (``src/Alpacc/Lexer/RegularExpression.hs:55-61``)."""
    tag = r[0]
    if tag == "eps" or tag == "star":
        return True
    if tag in ("lit", "range"):
        return False
    if tag == "alt":
        return produces_epsilon(r[1]) or produces_epsilon(r[2])
    return produces_epsilon(r[1]) and produces_epsilon(r[2])


class _Src:
    """Character cursor shared by the grammar and regex parsers."""

    def __init__(self, text: str, pos: int = 0):
        self.s = text
        self.i = pos

    def peek(self, n: int = 0) -> str:
        j = self.i + n
        return self.s[j] if j < len(self.s) else ""

    def startswith(self, lit: str) -> bool:
        return self.s.startswith(lit, self.i)

    def eof(self) -> bool:
        return self.i >= len(self.s)

    def error(self, what: str):
        line = self.s.count("\n", 0, self.i) + 1
        raise GrammarError("parse error at line %d: expected %s" % (line, what))

    # whitespace inside regexes: plain space1, no comments
    # (``src/Alpacc/Lexer/RegularExpression.hs:81-85``)
    def rx_space(self):
        while not self.eof() and _is_space(self.peek()):
            self.i += 1

    # whitespace in the grammar: space1 and '#' line comments
    # (``src/Alpacc/CFG.hs:174-178``)
    def g_space(self):
        while not self.eof():
            c = self.peek()
            if _is_space(c):
                self.i += 1
            elif c == "#":
                while not self.eof() and self.peek() != "\n":
                    self.i += 1
            else:
                break


def _utf8(ch: str) -> bytes:
    return ch.encode("utf-8", "surrogatepass")


def _rx_char(src: _Src) -> Optional[bytes]:
    """``pChar`` (``src/Alpacc/Lexer/RegularExpression.hs:141-148``): escape,
    ``\\uHEX``, ``\\xHH`` byte, or a printable non-space non-operator char."""
    c = src.peek()
    if c == "\\":
        n = src.peek(1)
        if n in _ESCAPES:
            src.i += 2
            src.rx_space()
            return _utf8(_ESCAPES[n])
        if n == "u":
            j = src.i + 2
            k = j
            while k < len(src.s) and src.s[k] in "0123456789abcdefABCDEF":
                k += 1
            if k > j:
                src.i = k
                src.rx_space()
                return _utf8(chr(int(src.s[j:k], 16)))
        if n == "x":
            h = src.s[src.i + 2: src.i + 4]
            if len(h) == 2 and all(x in "0123456789abcdefABCDEF" for x in h):
                src.i += 4
                src.rx_space()
                return bytes([int(h, 16)])
        return None
    if c and c not in _NOT_PRINT and _is_print(c) and not _is_space(c):
        src.i += 1
        src.rx_space()
        return _utf8(c)
    return None


def _rx_byte(src: _Src) -> Optional[int]:
    if src.peek() == "\\" and src.peek(1) == "x":
        h = src.s[src.i + 2: src.i + 4]
        if len(h) == 2 and all(x in "0123456789abcdefABCDEF" for x in h):
            src.i += 4
            src.rx_space()
            return int(h, 16)
    return None


def _rx_alnum(src: _Src) -> Optional[str]:
    c = src.peek()
    if c and c.isalnum():
        src.i += 1
        src.rx_space()
        return c
    return None


def _rx_range(src: _Src):
    """``pRange`` (``src/Alpacc/Lexer/RegularExpression.hs:175-197``)."""
    src.i += 1  # '['
    src.rx_space()
    items: List[bytes] = []
    while True:
        save = src.i
        a = _rx_alnum(src)
        if a is not None and src.peek() == "-":
            src.i += 1
            src.rx_space()
            b = _rx_alnum(src)
            if b is not None:
                items.extend(_utf8(chr(x)) for x in range(ord(a), ord(b) + 1))
                continue
        src.i = save
        a = _rx_byte(src)
        if a is not None and src.peek() == "-":
            src.i += 1
            src.rx_space()
            b = _rx_byte(src)
            if b is not None:
                items.extend(bytes([x]) for x in range(a, b + 1))
                continue
        src.i = save
        a = _rx_byte(src)
        if a is not None:
            items.append(bytes([a]))
            continue
        src.i = save
        a = _rx_alnum(src)
        if a is not None:
            items.append(_utf8(a))
            continue
        src.i = save
        break
    if not items:
        src.error("range element")
    if src.peek() != "]":
        src.error("']'")
    src.i += 1
    src.rx_space()
    return ("range", tuple(items))


def _rx_term(src: _Src):
    """``pTerm`` with postfix ``* + ?`` (``RegularExpression.hs:199-215``)."""
    c = src.peek()
    if c == "[":
        term = _rx_range(src)
    elif c == "(":
        src.i += 1
        src.rx_space()
        term = _rx_alter(src)
        if src.peek() != ")":
            src.error("')'")
        src.i += 1
        src.rx_space()
    else:
        lit = _rx_char(src)
        if lit is None:
            return None
        term = ("lit", lit)
    while True:
        c = src.peek()
        if c == "*":
            term = ("star", term)
        elif c == "+":
            term = ("cat", term, ("star", term))
        elif c == "?":
            term = ("alt", ("eps",), term)
        else:
            break
        src.i += 1
        src.rx_space()
    return term


def _rx_concat(src: _Src):
    r = ("eps",)
    while True:
        t = _rx_term(src)
        if t is None:
            return r
        r = ("cat", r, t)


def _rx_alter(src: _Src):
    r = _rx_concat(src)
    while src.peek() == "|":
        src.i += 1
        src.rx_space()
        r = ("alt", r, _rx_concat(src))
    return r


def parse_regex(text: str):
    """Parse a whole regex (``regExFromText``)."""
    src = _Src(text)
    r = _rx_alter(src)
    if not src.eof():
        src.error("end of regex")
    return r


# --------------------------------------------------------------------------
# .alp files
# --------------------------------------------------------------------------

@dataclass
class TRule:
    t: T
    regex: tuple


@dataclass
class NTRule:
    nt: NT
    name: Optional[str]
    rhs: List[Sym]


@dataclass
class CFG:
    lookback: int
    lookahead: int
    t_rules: List[TRule]
    nt_rules: List[NTRule]


def _ident(src: _Src, first) -> Optional[str]:
    c = src.peek()
    if not (c and c.isascii() and first(c)):
        return None
    j = src.i + 1
    while j < len(src.s) and (src.s[j] == "_" or (src.s[j].isascii() and src.s[j].isalnum())):
        j += 1
    name = src.s[src.i:j]
    src.i = j
    src.g_space()
    return name


def _lex_lit(src: _Src, lit: str) -> bool:
    if src.startswith(lit):
        src.i += len(lit)
        src.g_space()
        return True
    return False


def _decimal(src: _Src) -> Optional[int]:
    j = src.i
    while j < len(src.s) and src.s[j].isdigit() and src.s[j].isascii():
        j += 1
    if j == src.i:
        return None
    v = int(src.s[src.i:j])
    src.i = j
    src.g_space()
    return v


def parse_cfg(text: str) -> CFG:
    """``cfgFromText`` (``src/Alpacc/CFG.hs:226-235``)."""
    src = _Src(text)
    src.g_space()
    lookback, lookahead = 0, 1  # defaultParams (src/Alpacc/CFG.hs:68-73)
    save = src.i
    if _lex_lit(src, "params"):
        if not _lex_lit(src, "{"):
            src.i = save
        else:
            while True:
                key = None
                if _lex_lit(src, "lookback"):
                    key = "lookback"
                elif _lex_lit(src, "lookahead"):
                    key = "lookahead"
                if key is None:
                    break
                if not _lex_lit(src, "="):
                    src.error("'='")
                v = _decimal(src)
                if v is None:
                    src.error("decimal")
                if not _lex_lit(src, "."):
                    src.error("'.'")
                if key == "lookback":
                    lookback = v
                else:
                    lookahead = v
            if not _lex_lit(src, "}"):
                src.error("'}'")
    t_rules: List[TRule] = []
    while True:
        save = src.i
        name = _ident(src, str.islower)
        if name is None or not _lex_lit(src, "=") or not _lex_lit(src, "/"):
            src.i = save
            break
        regex = _rx_alter(src)
        if not _lex_lit(src, "/") or not _lex_lit(src, "."):
            src.i = save
            break
        t_rules.append(TRule(T(False, name), regex))
    nt_rules: List[NTRule] = []
    while not src.eof():
        nt = _ident(src, str.isupper)
        if nt is None:
            src.error("nonterminal rule")
        label = None
        if src.peek() == "[":
            src.i += 1
            src.g_space()
            label = _ident(src, str.isupper)
            if label is None:
                src.error("production name")
            if src.peek() != "]":
                src.error("']'")
            src.i += 1
            src.g_space()
        if not _lex_lit(src, "->"):
            src.error("'->'")
        alts: List[List[Sym]] = [[]]
        while True:
            c = src.peek()
            if c == '"':
                j = src.i + 1
                while j < len(src.s) and src.s[j] != '"' and _is_print(src.s[j]):
                    j += 1
                if j == src.i + 1 or j >= len(src.s) or src.s[j] != '"':
                    src.error("string literal")
                alts[-1].append(("t", T(True, src.s[src.i + 1:j])))
                src.i = j + 1
                src.g_space()
                continue
            name = _ident(src, str.islower)
            if name is not None:
                alts[-1].append(("t", T(False, name)))
                continue
            name = _ident(src, str.isupper)
            if name is not None:
                alts[-1].append(("n", NT(name)))
                continue
            if _lex_lit(src, "|"):
                alts.append([])
                continue
            break
        if not _lex_lit(src, "."):
            src.error("'.'")
        for rhs in alts:
            nt_rules.append(NTRule(NT(nt), label, rhs))
    return CFG(lookback, lookahead, t_rules, nt_rules)


# --------------------------------------------------------------------------
# Lexer spec: which regex belongs to which terminal, with what priority
# --------------------------------------------------------------------------

def _rule_terminals(cfg: CFG) -> List[T]:
    """``foldMap ruleTerminals ntRules`` as a sorted Set (``CFG.hs:108-113``)."""
    s = set()
    for r in cfg.nt_rules:
        for kind, v in r.rhs:
            if kind == "t":
                s.add(v)
    return sorted(s)


def lexer_spec(cfg: CFG) -> Tuple[Dict[T, int], Dict[T, tuple]]:
    """``cfgToDFALexerSpec`` (``src/Alpacc/CFG.hs:146-170``).

    Returns ``(order, regex)``: terminal -> priority (lower wins on ties,
    ``src/Alpacc/Lexer/DFA.hs:371-384``) and terminal -> regex.  Implicit
    literal rules come first, then the declared rules in file order."""
    declared = [r.t for r in cfg.t_rules]
    implicit = []
    for t in _rule_terminals(cfg):
        if t in declared:
            continue
        if not t.lit:
            raise GrammarError("Can not create literal from: %s" % t.name)
        rx = None
        for ch in t.name:
            lit = ("lit", _utf8(ch))
            rx = lit if rx is None else ("cat", rx, lit)
        implicit.append((t, rx))
    rules = implicit + [(r.t, r.regex) for r in cfg.t_rules]
    for t, rx in rules:
        if produces_epsilon(rx):
            raise GrammarError("Error: %s may not produce empty strings." % t.pretty())
    if not rules:
        raise GrammarError("CFG has no lexical rules.")
    order: Dict[T, int] = {}
    regex: Dict[T, tuple] = {}
    for i, (t, rx) in enumerate(rules):
        order[t] = i
        regex[t] = rx
    return order, regex


# --------------------------------------------------------------------------
# Parsing grammar and symbol encoding
# --------------------------------------------------------------------------

# Augmented terminal ids in the parsing grammar, as Python values:
#   ('used', T) | ('unused',) | ('rts',) [RightTurnstile, '⊢'] | ('lts',) ['⊣']
# Augmented nonterminals:
#   ('wrap', T)  -- AugmentedNonterminal (Terminal t), the per-terminal wrapper
#   ('nt', NT)   -- AugmentedNonterminal (Nonterminal nt)
#   ('start',)   -- Start


@dataclass
class ParsingGrammar:
    terminals: List[tuple]            # augmented terminals, grammar order
    nonterminals: List[tuple]         # augmented nonterminals, grammar order
    productions: List[Tuple[tuple, List[tuple]]]  # (lhs, rhs); rhs items ('t', aterm) | ('n', ant)
    start: tuple
    names: Dict[int, str]             # production index -> label from the file
    grammar_terminals: List[T]        # terminals before augmentation


def _closure_productive(nts, prods) -> set:
    prod = set()
    while True:
        new = set(prod)
        for lhs, rhs in prods:
            if all(k == "t" or v in prod for k, v in rhs):
                new.add(lhs)
        if new == prod:
            return prod
        prod = new


def parsing_grammar(cfg: CFG) -> ParsingGrammar:
    """``cfgToGrammar`` + ``parsingGrammar`` (``src/Alpacc/CFG.hs:115-139``,
    ``src/Alpacc/Grammar.hs:393-398``)."""
    if not cfg.nt_rules:
        raise GrammarError("CFG has no production rules.")
    names = {i: r.name for i, r in enumerate(cfg.nt_rules) if r.name is not None}
    nts: List[NT] = []
    for r in cfg.nt_rules:
        if r.nt not in nts:
            nts.append(r.nt)
    start = cfg.nt_rules[0].nt
    terminals: List[T] = []
    for t in [r.t for r in cfg.t_rules] + _rule_terminals(cfg):
        if t not in terminals:
            terminals.append(t)
    prods = [(r.nt, list(r.rhs)) for r in cfg.nt_rules]
    # grammarError (src/Alpacc/Grammar.hs:281-295)
    seen = set()
    for lhs, rhs in prods:
        key = (lhs, tuple(rhs))
        if key in seen:
            raise GrammarError("The given grammar contains duplicate productions.")
        seen.add(key)
    nonprod = set(nts) - _closure_productive(nts, prods)
    if nonprod:
        raise GrammarError(
            "The given grammar contains nonproductive productions due to the "
            "following nonterminals %s." % ", ".join(sorted(n.name for n in nonprod)))
    # extendByTerminals: every terminal occurrence becomes its wrapper NT
    a_prods: List[Tuple[tuple, List[tuple]]] = []
    for lhs, rhs in prods:
        new_rhs = [("n", ("wrap", v)) if k == "t" else ("n", ("nt", v)) for k, v in rhs]
        a_prods.append((("nt", lhs), new_rhs))
    for t in terminals:
        a_prods.append((("wrap", t), [("t", ("used", t))]))
    a_prods.append((("start",), [("t", ("rts",)), ("n", ("nt", start)), ("t", ("lts",))]))
    a_terms = [("used", t) for t in terminals] + [("unused",), ("rts",), ("lts",)]
    a_nts = [("wrap", t) for t in terminals] + [("nt", n) for n in nts] + [("start",)]
    return ParsingGrammar(a_terms, a_nts, a_prods, ("start",), names, terminals)


IGNORE = T(False, "ignore")


def encode_symbols(pg: ParsingGrammar) -> Dict[tuple, int]:
    """``encodeSymbols`` (``src/Alpacc/Encode.hs:122-146``): ordinary terminals
    in grammar order, then ignore, Unused, ⊢, ⊣, then every nonterminal.
    Keys are ('t', aterm) / ('n', ant)."""
    special = {("used", IGNORE), ("unused",), ("rts",), ("lts",)}
    fts = [t for t in pg.terminals if t not in special]
    order = fts
    for s in [("used", IGNORE), ("unused",), ("rts",), ("lts",)]:
        if s in pg.terminals:
            order = order + [s]
    syms = [("t", t) for t in order] + [("n", n) for n in pg.nonterminals]
    return {s: i for i, s in enumerate(syms)}


def encode_lexer_terminals(order: Dict[T, int]) -> Dict[tuple, int]:
    """``encodeTerminals`` over ``dfaTerminals`` for lexer-only mode
    (``src/Alpacc/Encode.hs:148-162``, ``src/Alpacc/Generator/Analyzer.hs:106-110``):
    terminals sorted by ``Ord T`` excluding ignore, then ignore, then Unused."""
    ts = sorted(order.keys())
    fts = [("used", t) for t in ts if t != IGNORE]
    tail = ([("used", IGNORE)] if IGNORE in ts else []) + [("unused",)]
    return {s: i for i, s in enumerate(fts + tail)}


def terminal_names(enc: Dict[tuple, int]) -> List[str]:
    """``nameTerminals`` (``src/Alpacc/Generator/Analyzer.hs:97-104``)."""
    out = [""] * len(enc)
    for s, i in enc.items():
        if s[0] == "used":
            out[i] = s[1].name if not s[1].lit else "literal_%d" % i
        else:
            out[i] = "empty_%d" % i
    return out


def production_names(pg: ParsingGrammar) -> List[str]:
    """``productionNames`` with ``nameProduction`` (``src/Alpacc/Encode.hs:344-351``,
    ``src/Alpacc/Generator/Analyzer.hs:140-147``)."""
    out = []
    for i, (lhs, _rhs) in enumerate(pg.productions):
        if i in pg.names:
            out.append(pg.names[i])
        elif lhs[0] == "start":
            out.append("start_%d" % i)
        elif lhs[0] == "nt":
            out.append("%s_%d" % (lhs[1].name, i))
        elif not lhs[1].lit:
            out.append("%s_%d" % (lhs[1].name, i))
        else:
            out.append("Literal_%d" % i)
    return out
