"""ORACLE build recipe — translate the reference's fixed-form Fortran 77 ordering
routines to C so that they can be compiled and executed here (no Fortran
compiler is installed).  Test infrastructure only.

It handles exactly the subset those files use (the MMD routines src/ordmmd.F,
genmmd.F, mmdint.F, mmdelm.F, mmdupd.F, mmdnum.F, the RCM routines genrcm.F,
rcm.F, fnroot.F, rootls.F, degree.F and the AMD routine amdbar.F):
`#if MMDIDXSIZE` / `RCMIDXSIZE` / `AMDIDXSIZE` blocks (the 32-bit branch is kept,
as in the reference's default build, src/CMakeLists.txt:138-154), INTEGER
declarations of scalars and 1-D arrays, INTRINSIC, assignments, logical IF with a
single statement, IF (...) THEN / ELSE IF (...) THEN / ELSE / ENDIF, GO TO,
labelled CONTINUE, DO loops with a terminal label, the intrinsics MAX, MIN, MOD
and ABS of two (one) integer arguments, CALL, RETURN and END.  Fortran semantics preserved: arguments by reference,
1-based arrays, blanks insignificant, DO trip counts fixed at loop entry.

    python oracle/f77_to_c.py OUT.c FILE.F [FILE.F ...]
"""
from __future__ import annotations

import re
import sys

INTRINSICS = {"max", "min", "mod", "abs"}
OPS = [(".lt.", " < "), (".le.", " <= "), (".gt.", " > "), (".ge.", " >= "), (".eq.", " == "),
       (".ne.", " != "), (".and.", " && "), (".or.", " || "), (".not.", " !")]


def preprocess(text: str, mmdidxsize: int = 32) -> list[str]:
    """Keep the branch of `#if MMDIDXSIZE == 64 / #else / #endif` for the given size."""
    out, stack = [], []
    for line in text.splitlines():
        s = line.strip().replace(" ", "")
        if s.startswith("#if"):
            m = re.match(r"#if(?:MMD|RCM|AMD)IDXSIZE==(\d+)", s)
            if not m:
                raise ValueError(f"unsupported directive: {line}")
            stack.append(int(m.group(1)) == mmdidxsize)
            continue
        if s.startswith("#else"):
            stack[-1] = not stack[-1]
            continue
        if s.startswith("#endif"):
            stack.pop()
            continue
        if s.startswith("#"):
            raise ValueError(f"unsupported directive: {line}")
        if all(stack):
            out.append(line)
    return out


def statements(lines: list[str]) -> list[tuple[str | None, str]]:
    """Fixed form: (label, statement text) with continuations joined and blanks removed."""
    stmts: list[list] = []
    for raw in lines:
        line = raw.expandtabs(6).rstrip("\n")
        if not line.strip() or line[0] in "cC*!":
            continue
        line = line[:72]
        cont = len(line) > 5 and line[5] not in " 0" and not line[:5].strip()
        body = line[6:] if len(line) > 6 else ""
        if cont:
            stmts[-1][1] += body
        else:
            lab = line[:5].strip() or None
            stmts.append([lab, body])
    return [(lab, re.sub(r"\s+", "", txt).lower()) for lab, txt in stmts]


def split_top(s: str, sep: str = ",") -> list[str]:
    """Split at separators outside parentheses."""
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return parts


def match_paren(s: str, i: int) -> int:
    """Index of the ')' matching the '(' at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    raise ValueError(f"unbalanced parentheses: {s}")


class Subroutine:
    def __init__(self, name: str, args: list[str]):
        self.name = name
        self.args = args
        self.arrays: set[str] = set()
        self.scalars: set[str] = set()
        self.body: list[str] = []
        self.open_do: list[str] = []   # terminal labels of open DO loops
        self.ntemp = 0

    # -- expressions --------------------------------------------------------
    def expr(self, s: str) -> str:
        for f, t in OPS:
            s = s.replace(f, t)
        out, i = "", 0
        while i < len(s):
            m = re.match(r"[a-z][a-z0-9_]*", s[i:])
            if m and (i == 0 or not (s[i - 1].isalnum() or s[i - 1] == "_")):
                name = m.group(0)
                j = i + len(name)
                if j < len(s) and s[j] == "(" and name in self.arrays:
                    k = match_paren(s, j)
                    out += f"{name}[({self.expr(s[j + 1:k])}) - 1]"
                    i = k + 1
                    continue
                if j < len(s) and s[j] == "(" and name in INTRINSICS:
                    k = match_paren(s, j)
                    out += f"f_{name}(" + ", ".join(self.expr(a) for a in split_top(s[j + 1:k])) + ")"
                    i = k + 1
                    continue
                if name in self.args and name not in self.arrays:
                    out += f"(*{name})"
                else:
                    out += name
                i = j
                continue
            out += s[i]
            i += 1
        return out

    def actual(self, a: str, pre: list[str]) -> str:
        """Actual argument passed by reference."""
        m = re.fullmatch(r"([a-z][a-z0-9_]*)", a)
        if m:
            name = m.group(1)
            if name in self.arrays or name in self.args:
                return name
            return f"&{name}"
        m = re.fullmatch(r"([a-z][a-z0-9_]*)\((.*)\)", a)
        if m and m.group(1) in self.arrays:
            return f"&{m.group(1)}[({self.expr(m.group(2))}) - 1]"
        self.ntemp += 1
        t = f"_t{self.ntemp}"
        pre.append(f"int {t} = {self.expr(a)};")
        return f"&{t}"

    # -- statements ---------------------------------------------------------
    def stmt(self, s: str) -> str:
        if s == "return":
            return "return;"
        if s == "continue":
            return ";"
        m = re.fullmatch(r"goto(\d+)", s)
        if m:
            return f"goto L{m.group(1)};"
        if s.startswith("if("):
            k = match_paren(s, 2)
            return f"if ({self.expr(s[3:k])}) {{ {self.stmt(s[k + 1:])} }}"
        if s.startswith("call"):
            m = re.fullmatch(r"call([a-z][a-z0-9_]*)\((.*)\)", s)
            pre: list[str] = []
            acts = [self.actual(a, pre) for a in split_top(m.group(2))]
            return "{ " + " ".join(pre) + f" {m.group(1)}_({', '.join(acts)}); }}"
        lhs, rhs = split_top(s, "=")[0], "=".join(split_top(s, "=")[1:])
        if not rhs:
            raise ValueError(f"unsupported statement: {s}")
        return f"{self.expr(lhs)} = {self.expr(rhs)};"

    def add(self, label: str | None, s: str) -> None:
        m = re.fullmatch(r"do(\d+)([a-z][a-z0-9_]*)=(.*)", s)
        if m:
            lab, var = m.group(1), m.group(2)
            lo, hi = split_top(m.group(3))
            if label:
                self.body.append(f"L{label}: ;")
            v = self.expr(var)
            self.body.append(f"{{ int _trip{lab} = ({self.expr(hi)}) - ({self.expr(lo)}) + 1; "
                             f"for ({v} = {self.expr(lo)}; _trip{lab} > 0; --_trip{lab}, ++{v}) {{")
            self.open_do.append(lab)
            return
        if s.startswith("if(") and s.endswith("then") and match_paren(s, 2) == len(s) - 5:
            if label:
                self.body.append(f"L{label}: ;")
            self.body.append(f"if ({self.expr(s[3:-5])}) {{")
            return
        m = re.fullmatch(r"elseif(\(.*\))then", s)
        if m and match_paren(s, 6) == len(s) - 5:
            if label:
                raise ValueError(f"labelled ELSE IF: {s}")
            self.body.append(f"}} else if ({self.expr(s[7:-5])}) {{")
            return
        if s == "else":
            if label:
                raise ValueError(f"labelled ELSE: {s}")
            self.body.append("} else {")
            return
        if s in ("endif", "endif;"):
            if label:
                self.body.append(f"L{label}: ;")
            self.body.append("}")
            return
        if label and label in self.open_do:
            self.body.append(f"  {self.stmt(s)}")
            self.body.append(f"L{label}: ;")
            while self.open_do and self.open_do[-1] == label:
                self.open_do.pop()
                self.body.append("} }")
            return
        if label:
            self.body.append(f"L{label}: ;")
        self.body.append(f"  {self.stmt(s)}")

    def declare(self, s: str) -> None:
        decl = re.sub(r"^integer(\*\d+)?", "", s)
        for item in split_top(decl):
            m = re.fullmatch(r"([a-z][a-z0-9_]*)(\(.*\))?", item)
            if not m:
                raise ValueError(f"bad declaration: {s}")
            (self.arrays if m.group(2) else self.scalars).add(m.group(1))

    def emit(self) -> str:
        params = ", ".join(f"int* {a}" for a in self.args)
        locals_ = sorted((self.scalars | self.arrays) - set(self.args))
        if any(l in self.arrays for l in locals_):
            raise ValueError("local arrays are not supported")
        head = f"void {self.name}_({params}) {{\n"
        decl = f"  int {', '.join(locals_)};\n" if locals_ else ""
        return head + decl + "\n".join(self.body) + "\n}\n"


def translate(paths: list[str], skip: frozenset = frozenset({"perm_inverse"})) -> str:
    """C for the subroutines of the given files; subroutines named in `skip` (helpers the
    path does not call, e.g. perm_inverse at the end of genrcm.F) are left out."""
    subs: list[Subroutine] = []
    for p in paths:
        cur = None
        skipping = False
        for label, s in statements(preprocess(open(p).read())):
            if skipping:
                skipping = s != "end"
                continue
            if s.startswith("subroutine"):
                m = re.fullmatch(r"subroutine([a-z][a-z0-9_]*)\((.*)\)", s)
                if m.group(1) in skip:
                    skipping = True
                    continue
                cur = Subroutine(m.group(1), split_top(m.group(2)))
                subs.append(cur)
            elif re.match(r"integer(\*\d+)?[a-z]", s):
                cur.declare(s)
            elif s.startswith("intrinsic"):
                continue
            elif s == "end":
                if cur.open_do:
                    raise ValueError(f"unterminated DO in {cur.name}")
                cur = None
            else:
                cur.add(label, s)
    protos = "".join(f"void {s.name}_({', '.join('int*' for _ in s.args)});\n" for s in subs)
    banner = ("/* Generated from the reference's Fortran sources by oracle/f77_to_c.py.\n"
              " * Oracle infrastructure: not part of the product. */\n"
              "static int iabs(int x) { return x < 0 ? -x : x; }  /* Fortran IABS */\n"
              "static int f_abs(int x) { return x < 0 ? -x : x; }\n"
              "static int f_max(int a, int b) { return a > b ? a : b; }\n"
              "static int f_min(int a, int b) { return a < b ? a : b; }\n"
              "static int f_mod(int a, int b) { return a % b; }  /* Fortran MOD: sign of a */\n")
    return banner + protos + "\n" + "\n".join(s.emit() for s in subs)


if __name__ == "__main__":
    out, srcs = sys.argv[1], sys.argv[2:]
    with open(out, "w") as f:
        f.write(translate(srcs))
