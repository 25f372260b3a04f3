"""Render the reference's ``src/opt_sell_c_sigma.cpp.mako`` without Mako.

TEST INFRASTRUCTURE ONLY (oracle build). The template has one loop
(``%for C in range(2, 18, 2)``) and one ``%if target_os == 'windows_arm64ec'``
block; the oracle build selects the Arm64EC configuration (``-D__arm64ec__``),
under which the reference uses its portable C++ SELL kernels for float and
double, so the ``%if`` block is kept. The rendered file is written under
``oracle/_ref/`` (git-ignored) and never committed.

Usage: python render_opt_scs.py <template> <output>
"""
import re
import sys


def render(text: str) -> str:
    out = []
    lines = text.splitlines()
    i = 0
    while i < len(lines):
        line = lines[i]
        s = line.strip()
        m = re.match(r"%for\s+(\w+)\s+in\s+range\((\d+),\s*(\d+),\s*(\d+)\):", s)
        if m:
            var, a, b, step = m.group(1), int(m.group(2)), int(m.group(3)), int(m.group(4))
            body = []
            i += 1
            while lines[i].strip() != "%endfor":
                body.append(lines[i])
                i += 1
            for v in range(a, b, step):
                for bl in body:
                    out.append(bl.replace("${" + var + "}", str(v)))
            i += 1
            continue
        if s.startswith("%if") or s.startswith("%endif"):
            i += 1
            continue
        out.append(line)
        i += 1
    return "\n".join(out) + "\n"


if __name__ == "__main__":
    src, dst = sys.argv[1], sys.argv[2]
    with open(src) as f:
        txt = f.read()
    with open(dst, "w") as f:
        f.write(render(txt))
