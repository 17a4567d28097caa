"""Regex front end: pattern -> Thompson NFA -> subset DFA -> minimal complete DFA.

Drop-in for the reference module ``src/regex_to_dfa.py``; the public names
(``EPSILON``, ``NFAState``, ``NFA``, ``RegexParser``, ``DFA``,
``epsilon_closure``, ``nfa_to_dfa``, ``complete_dfa``, ``minimize_dfa``,
``compile_regex``) and their fields match it (reference
src/regex_to_dfa.py:15-39, 99-118, 215-233, 236-376).

Accepted syntax (reference src/regex_to_dfa.py:122-210): concatenation,
``|``, postfix ``* + ?`` (one per atom; a second postfix operator is read as
a literal), ``( )``, ``.`` (the 95 printable ASCII characters), classes
``[abc] [a-z] [^...]`` (negation is taken against the 95 printable
characters, an empty class matches ``\\x00``), escapes ``\\d \\w \\s`` and
``\\<char>`` for a literal. Parsing stops at an unmatched ``)``.

NFA states are created in textbook Thompson order (two fresh states per
literal / alternation / closure operator), so the state ids, and hence the
``NFAMatrices`` built from them, equal the reference's. DFA states are
numbered canonically (breadth-first from the start over the sorted
alphabet), which makes final-state ids reproducible across processes; the
reference numbers them in Python set order, so for regex-built DFAs parity
is defined on the language (accept flags), not on state ids.
"""

from __future__ import annotations

import string
from collections import deque
from dataclasses import dataclass, field
from typing import Optional

EPSILON = None

_PRINTABLE = string.printable[:95]
_DIGITS = "0123456789"
_WORD = string.ascii_letters + string.digits + "_"
_SPACE = " \t\n\r"


@dataclass
class NFAState:
    id: int
    transitions: dict = field(default_factory=dict)  # symbol (or None) -> list[int]
    is_accept: bool = False


class NFA:
    """Epsilon-NFA with integer state ids and ``None`` as the epsilon label."""

    def __init__(self):
        self.states: dict[int, NFAState] = {}
        self.start: int = -1
        self.accept: int = -1
        self.alphabet: set[str] = set()
        self._next_id = 0

    def new_state(self, is_accept: bool = False) -> int:
        sid = self._next_id
        self._next_id += 1
        self.states[sid] = NFAState(id=sid, is_accept=is_accept)
        return sid

    def add_trans(self, src: int, sym: Optional[str], dst: int) -> None:
        self.states[src].transitions.setdefault(sym, []).append(dst)
        if sym is not None:
            self.alphabet.add(sym)


# A fragment is (entry state, exit state).
Fragment = tuple[int, int]


class RegexParser:
    """Recursive-descent parser that emits Thompson fragments into ``self.nfa``."""

    def __init__(self, pattern: str):
        self.pattern = pattern
        self.pos = 0
        self.nfa = NFA()

    # -- small helpers ----------------------------------------------------
    def _peek(self) -> Optional[str]:
        return self.pattern[self.pos] if self.pos < len(self.pattern) else None

    def _take(self) -> str:
        ch = self.pattern[self.pos]
        self.pos += 1
        return ch

    def _pair(self) -> Fragment:
        a = self.nfa.new_state()
        b = self.nfa.new_state()
        return a, b

    def _symbol(self, ch: str) -> Fragment:
        a, b = self._pair()
        self.nfa.add_trans(a, ch, b)
        return a, b

    def _empty(self) -> Fragment:
        a, b = self._pair()
        self.nfa.add_trans(a, EPSILON, b)
        return a, b

    def _union(self, frags: list[Fragment]) -> Fragment:
        a, b = self._pair()
        for f_in, f_out in frags:
            self.nfa.add_trans(a, EPSILON, f_in)
            self.nfa.add_trans(f_out, EPSILON, b)
        return a, b

    def _union_of_chars(self, chars) -> Fragment:
        return self._union([self._symbol(c) for c in chars])

    # -- grammar ------------------------------------------------------------
    def parse(self) -> NFA:
        f_in, f_out = self._alternation()
        self.nfa.start = f_in
        self.nfa.accept = f_out
        self.nfa.states[f_out].is_accept = True
        return self.nfa

    def _alternation(self) -> Fragment:
        options = [self._sequence()]
        while self._peek() == "|":
            self._take()
            options.append(self._sequence())
        return options[0] if len(options) == 1 else self._union(options)

    def _sequence(self) -> Fragment:
        items: list[Fragment] = []
        while self._peek() not in (None, "|", ")"):
            items.append(self._postfix())
        if not items:
            return self._empty()
        head, tail = items[0]
        for f_in, f_out in items[1:]:
            self.nfa.add_trans(tail, EPSILON, f_in)
            tail = f_out
        return head, tail

    def _postfix(self) -> Fragment:
        body_in, body_out = self._atom()
        op = self._peek()
        if op not in ("*", "+", "?"):
            return body_in, body_out
        self._take()
        a, b = self._pair()
        add = self.nfa.add_trans
        add(a, EPSILON, body_in)
        if op != "+":                       # '*' and '?' may skip the body
            add(a, EPSILON, b)
        if op != "?":                       # '*' and '+' may repeat the body
            add(body_out, EPSILON, body_in)
        add(body_out, EPSILON, b)
        return a, b

    def _atom(self) -> Fragment:
        ch = self._peek()
        if ch == "(":
            self._take()
            inner = self._alternation()
            if self._peek() == ")":
                self._take()
            return inner
        if ch == "[":
            return self._char_class()
        if ch == ".":
            self._take()
            return self._union_of_chars(_PRINTABLE)
        if ch == "\\":
            self._take()
            esc = self._take()
            named = {"d": _DIGITS, "w": _WORD, "s": _SPACE}.get(esc)
            if named is not None:
                return self._union_of_chars(named)
            return self._symbol(esc)
        self._take()
        return self._symbol(ch)

    def _char_class(self) -> Fragment:
        self._take()  # '['
        members: list[str] = []
        negated = False
        if self._peek() == "^":
            negated = True
            self._take()
        while self._peek() not in (None, "]"):
            lo = self._take()
            is_range = (self._peek() == "-" and self.pos + 1 < len(self.pattern)
                        and self.pattern[self.pos + 1] != "]")
            if is_range:
                self._take()
                hi = self._take()
                members.extend(chr(o) for o in range(ord(lo), ord(hi) + 1))
            else:
                members.append(lo)
        if self._peek() == "]":
            self._take()
        if negated:
            members = list(set(_PRINTABLE) - set(members))
        if not members:
            members = ["\x00"]
        if len(members) == 1:
            return self._symbol(members[0])
        return self._union_of_chars(members)


# ---------------------------------------------------------------------------
# DFA
# ---------------------------------------------------------------------------

@dataclass
class DFA:
    n_states: int
    start: int
    accept_states: set[int]
    transitions: dict[int, dict[str, int]]
    alphabet: set[str]
    dead_state: Optional[int] = None

    def simulate(self, input_str: str) -> bool:
        """Sequential walk. A symbol with no transition goes to the dead state
        when there is one, otherwise the string is rejected
        (reference src/regex_to_dfa.py:224-233)."""
        state = self.start
        delta = self.transitions
        for ch in input_str:
            row = delta.get(state, {})
            nxt = row.get(ch)
            if nxt is None:
                if self.dead_state is None:
                    return False
                nxt = self.dead_state
            state = nxt
        return state in self.accept_states

    def final_state(self, input_str: str) -> Optional[int]:
        """State reached after ``input_str`` under the same rules as
        :meth:`simulate`; ``None`` when the walk rejects early."""
        state = self.start
        for ch in input_str:
            nxt = self.transitions.get(state, {}).get(ch)
            if nxt is None:
                if self.dead_state is None:
                    return None
                nxt = self.dead_state
            state = nxt
        return state


def epsilon_closure(nfa: NFA, states) -> frozenset[int]:
    seen = set(states)
    todo = list(seen)
    while todo:
        s = todo.pop()
        for t in nfa.states[s].transitions.get(EPSILON, ()):
            if t not in seen:
                seen.add(t)
                todo.append(t)
    return frozenset(seen)


def nfa_to_dfa(nfa: NFA) -> DFA:
    """Subset construction; DFA state ids are assigned in BFS order over the
    sorted alphabet. Missing transitions are left undefined (see
    :func:`complete_dfa`)."""
    symbols = sorted(nfa.alphabet)
    first = epsilon_closure(nfa, [nfa.start])
    ids = {first: 0}
    order = [first]
    delta: dict[int, dict[str, int]] = {}
    queue = deque([first])
    while queue:
        cur = queue.popleft()
        cid = ids[cur]
        row: dict[str, int] = {}
        for ch in symbols:
            moved = set()
            for s in cur:
                moved.update(nfa.states[s].transitions.get(ch, ()))
            if not moved:
                continue
            nxt = epsilon_closure(nfa, moved)
            if nxt not in ids:
                ids[nxt] = len(order)
                order.append(nxt)
                queue.append(nxt)
            row[ch] = ids[nxt]
        delta[cid] = row
    accepting = {ids[S] for S in order if nfa.accept in S}
    return DFA(n_states=len(order), start=0, accept_states=accepting,
               transitions=delta, alphabet=set(nfa.alphabet))


def complete_dfa(dfa: DFA) -> DFA:
    """Add one absorbing dead state when some transition is undefined;
    otherwise clear ``dead_state`` (reference src/regex_to_dfa.py:279-299)."""
    missing = any(ch not in dfa.transitions.get(s, {})
                  for s in range(dfa.n_states) for ch in dfa.alphabet)
    if not missing:
        dfa.dead_state = None
        return dfa
    dead = dfa.n_states
    dfa.n_states += 1
    dfa.dead_state = dead
    for s in range(dfa.n_states):
        row = dfa.transitions.setdefault(s, {})
        for ch in dfa.alphabet:
            row.setdefault(ch, dead)
    return dfa


def minimize_dfa(dfa: DFA) -> DFA:
    """Moore partition refinement on a complete DFA, then canonical BFS
    renumbering. Like the reference (src/regex_to_dfa.py:302-305), a DFA whose
    states are all accepting or all rejecting is returned unchanged."""
    n = dfa.n_states
    if not dfa.accept_states or len(dfa.accept_states) == n:
        return dfa
    symbols = sorted(dfa.alphabet)
    block = [1 if s in dfa.accept_states else 0 for s in range(n)]
    n_blocks = 2
    while True:
        signature = {}
        new_block = [0] * n
        for s in range(n):
            row = dfa.transitions.get(s, {})
            key = (block[s],) + tuple(block[row[ch]] if ch in row else -1 for ch in symbols)
            new_block[s] = signature.setdefault(key, len(signature))
        if len(signature) == n_blocks:
            break
        block, n_blocks = new_block, len(signature)
    # BFS renumbering of the quotient automaton from the start block.
    rep = {}
    for s in range(n):
        rep.setdefault(block[s], s)
    ids = {block[dfa.start]: 0}
    queue = deque([block[dfa.start]])
    delta: dict[int, dict[str, int]] = {}
    while queue:
        b = queue.popleft()
        row = dfa.transitions.get(rep[b], {})
        out = {}
        for ch in symbols:
            if ch not in row:
                continue
            tb = block[row[ch]]
            if tb not in ids:
                ids[tb] = len(ids)
                queue.append(tb)
            out[ch] = ids[tb]
        delta[ids[b]] = out
    # Blocks unreachable from the start are dropped; they cannot affect the language.
    accepting = {ids[block[s]] for s in dfa.accept_states if block[s] in ids}
    dead = None
    if dfa.dead_state is not None and block[dfa.dead_state] in ids:
        dead = ids[block[dfa.dead_state]]
    return DFA(n_states=len(ids), start=0, accept_states=accepting,
               transitions=delta, alphabet=set(dfa.alphabet), dead_state=dead)


def compile_regex(pattern: str, minimize: bool = True) -> DFA:
    """Pattern -> complete DFA (minimal when ``minimize``), as in the reference
    pipeline parse -> subset -> complete -> minimise -> complete
    (reference src/regex_to_dfa.py:356-364)."""
    nfa = RegexParser(pattern).parse()
    dfa = complete_dfa(nfa_to_dfa(nfa))
    if minimize:
        dfa = complete_dfa(minimize_dfa(dfa))
    return dfa
