#!/usr/bin/env python3
"""TEST INFRASTRUCTURE ONLY (oracle).

Rewrites one of the reference's HLSL compute shaders into C++ that compiles
against oracle/hlsl_shim.h, so the reference's own shader code can run on the
CPU as a second, independent check of the oracle restatement.  The output goes
to oracle/_ref/ (git-ignored); nothing of the reference is committed.

Every rewrite is token level and changes no arithmetic:

  1. comments removed;
  2. attributes removed: [numthreads(...)], [[vk::...]], [unroll]/[loop]/...;
  3. register / semantic annotations removed (": register(t1, space0)",
     ": SV_DispatchThreadID");
  4. the cbuffer block is unwrapped: its fields become globals, which is how
     HLSL code names them;
  5. parameter qualifiers: "out T x" / "inout T x" -> "T &x",
     "const in T x" -> "const T &x", "in T x" -> "T x";
  6. swizzle reads become calls: ".xyz" -> ".xyz()" (also .rgb .xy .zw), and
     the colour alias ".a" reads ".w";
  7. file-scope "static T x;" becomes thread_local (the RNG state `seed` is
     per invocation in HLSL; per host thread here);
  8. a statement with two or more Random() calls gets its calls hoisted into
     temporaries in textual order, since C++ leaves the evaluation order of
     operands and constructor arguments unspecified and the shader's stream
     order is left to right;
  9. "row_major" is dropped (the shim's float4x4 is row-major), "(T)0"
     becomes "T{}" and a scalar's ".xxx" becomes "float3(...)";
 10. optional instrumentation (--instrument): extra fields on the Hit struct
     that record the winning triangle and object slot, which the shader keeps
     only in locals.  Each anchor must match exactly once.

Usage: hlsl2cpp.py SRC.hlsl OUT.inc [--instrument hybrid|deferred]
"""
import re
import sys


def strip_comments(s: str) -> str:
    out, i, n = [], 0, len(s)
    while i < n:
        if s.startswith("//", i):
            j = s.find("\n", i)
            i = n if j < 0 else j
        elif s.startswith("/*", i):
            j = s.find("*/", i + 2)
            seg = s[i:(n if j < 0 else j + 2)]
            out.append("\n" * seg.count("\n"))
            i = n if j < 0 else j + 2
        else:
            out.append(s[i])
            i += 1
    return "".join(out)


def unwrap_cbuffer(s: str) -> str:
    m = re.search(r"\bcbuffer\s+\w+\s*\{", s)
    while m:
        depth, i = 1, m.end()
        while depth:
            if s[i] == "{":
                depth += 1
            elif s[i] == "}":
                depth -= 1
            i += 1
        body = s[m.end():i - 1]
        tail = i
        if s[tail:tail + 1] == ";":
            tail += 1
        s = s[:m.start()] + body + s[tail:]
        m = re.search(r"\bcbuffer\s+\w+\s*\{", s)
    return s


def hoist_random(s: str) -> str:
    calls = [m.start() for m in re.finditer(r"\bRandom\(\)", s)]
    # group calls by statement: no ; { } between consecutive calls
    groups, cur = [], []
    for c in calls:
        if cur and re.search(r"[;{}]", s[cur[-1]:c]):
            groups.append(cur)
            cur = []
        cur.append(c)
    if cur:
        groups.append(cur)
    counter = 0
    for g in reversed(groups):
        if len(g) < 2:
            continue
        start = max(s.rfind(";", 0, g[0]), s.rfind("{", 0, g[0]), s.rfind("}", 0, g[0])) + 1
        end = s.find(";", g[-1])
        stmt = s[start:end]
        if "?" in stmt or "&&" in stmt or "||" in stmt:
            raise SystemExit("hoist_random: conditional evaluation in a multi-Random statement")
        names = []
        new_stmt = stmt
        # replace from the back so offsets stay valid
        for k, c in reversed(list(enumerate(g))):
            name = f"ae_r{counter + k}"
            names.insert(0, name)
            rel = c - start
            new_stmt = new_stmt[:rel] + name + new_stmt[rel + len("Random()"):]
        decl = " ".join(f"const float {n} = Random();" for n in names)
        s = s[:start] + " " + decl + new_stmt + s[end:]
        counter += len(g)
    return s


def replace_once(s: str, anchor: str, new: str) -> str:
    if s.count(anchor) != 1:
        raise SystemExit(f"instrumentation anchor found {s.count(anchor)} times: {anchor!r}")
    return s.replace(anchor, new)


def instrument(s: str, kind: str) -> str:
    # The Hit struct gains the winner's triangle base, barycentrics and the
    # object slot; default member initialisers mark analytic hits.
    s = replace_once(s, "uint materialId;",
                     "uint materialId; uint aeTriBase = 0xFFFFFFFFu; float aeAlpha = 0.0f; "
                     "float aeBeta = 0.0f; uint aeObjSlot = 0xFFFFFFFFu;")
    if kind == "hybrid":
        s = replace_once(s, "hit.surface_uv = w0",
                         "hit.aeTriBase = bestBase; hit.aeAlpha = bestAlpha; hit.aeBeta = bestBeta; "
                         "hit.surface_uv = w0")
        s = replace_once(s, "far = h.Offset;", "h.aeObjSlot = node.Left + i; far = h.Offset;")
    return s


def transpile(src: str, kind: str | None) -> str:
    s = strip_comments(src)
    s = re.sub(r"\[\[vk::[^\]]*\]\]", "", s)
    s = re.sub(r"\[numthreads\([^)]*\)\]", "", s)
    s = re.sub(r"\[(unroll|loop|branch|flatten|fastopt)(\([^)]*\))?\]", "", s)
    s = re.sub(r":\s*register\([^)]*\)", "", s)
    s = re.sub(r":\s*SV_\w+", "", s)
    s = unwrap_cbuffer(s)
    s = re.sub(r"\brow_major\s+", "", s)
    s = re.sub(r"\((\w+)\)0\b", r"\1{}", s)                 # (Hit)0 -> Hit{}
    s = re.sub(r"\(([^()]*)\)\.xxx\b", r"float3(\1)", s)   # (scalar).xxx -> float3(scalar)
    s = re.sub(r"\bconst\s+in\s+(\w+)\s+(\w+)", r"const \1 &\2", s)
    s = re.sub(r"\binout\s+(\w+)\s+(\w+)", r"\1 &\2", s)
    s = re.sub(r"\bout\s+(\w+)\s+(\w+)", r"\1 &\2", s)
    s = re.sub(r"\bin\s+(\w+)\s+(\w+)", r"\1 \2", s)
    s = re.sub(r"\.(xyz|rgb|xy|zw)\b(?!\s*\()", r".\1()", s)
    s = re.sub(r"\.a\b(?!\s*\()", ".w", s)                  # colour alpha is the w member
    s = re.sub(r"(?m)^static\s+(?!const\b)(\w+)\s+(\w+)\s*;", r"static thread_local \1 \2;", s)
    s = hoist_random(s)
    if kind:
        s = instrument(s, kind)
    return s


def main(argv):
    if len(argv) < 3:
        print(__doc__)
        return 2
    kind = None
    if "--instrument" in argv:
        kind = argv[argv.index("--instrument") + 1]
    with open(argv[1]) as f:
        src = f.read()
    out = transpile(src, kind)
    with open(argv[2], "w") as f:
        f.write("// GENERATED by oracle/hlsl2cpp.py from " + argv[1].split("/")[-1] + "; do not commit.\n")
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
