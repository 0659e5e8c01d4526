"""The reference's option front end: ``-group.param v1 v2 ...`` on the command
line, or ``group.param v1 v2`` lines in a parameter file given as the first
non-dash argument (paramsParser.hxx:134-218).  The first definition of a key
wins and the command line is parsed before the file (paramsParser.hxx:208-209),
so the command line takes precedence.  A key given without a value reads as
true (paramsParser.hxx:340-341); ``-3`` is a value, not a key
(paramsParser.hxx:186).
"""
from __future__ import annotations

import re


class ParamsParser:
    def __init__(self, argv=None, fname="params.ini"):
        self._vals: dict[tuple[str, str], list[list[str]]] = {}
        argv = list(argv or [])
        i0 = 0
        if argv and not argv[0].startswith("-"):
            fname = argv[0]
            i0 = 1
        self._parse_args(argv[i0:])
        self.param_file = None
        try:
            with open(fname) as fh:
                self._parse_file(fh.read())
            self.param_file = fname
        except FileNotFoundError:
            if fname != "params.ini":
                raise ValueError(f"could not read parameter file '{fname}'")

    @staticmethod
    def _key(raw: str):
        if "." in raw:
            cat, what = raw.split(".", 1)
        else:
            cat, what = "default", raw
        return cat, what

    def _insert(self, raw, values):
        self._vals.setdefault(self._key(raw), []).append(list(values))

    def _parse_args(self, args):
        n = 0
        while n < len(args):
            a = args[n]
            if not a.startswith("-"):
                raise ValueError(f"ERROR parsing command line at: {a}")
            key = a[1:]
            n += 1
            vals = []
            while n < len(args) and (not args[n].startswith("-")
                                     or args[n][1:2].isdigit()):
                vals.append(args[n])
                n += 1
            self._insert(key, vals)

    def _parse_file(self, text):
        for line in text.splitlines():
            if "#" in line:
                line = line[: line.index("#")]
            toks = [t for t in re.split(r"[ =:{}\[\],\t]+", line) if t]
            if toks:
                self._insert(toks[0], toks[1:])

    def is_defined(self, what, cat):
        return len(self._vals.get((cat, what), []))

    def get(self, what, cat, default, which=-1, typ=None):
        """Value of cat.what (the which-th value of its first definition), or
        `default` when absent; converted to the type of `default`."""
        defs = self._vals.get((cat, what))
        if not defs:
            return default
        vals = defs[0]
        w = 0 if which < 0 else which
        if which >= 0 and len(vals) <= which:
            return default
        typ = typ or type(default)
        if not vals:
            return typ(True) if typ is not str else "1"
        s = vals[w]
        if typ is bool:
            try:
                return bool(int(s))
            except ValueError:
                return s.lower() in ("true", "yes")
        if typ is int:
            return int(float(s)) if re.fullmatch(r"[-+]?\d+(\.0*)?", s) else int(s)
        return typ(s)
