"""ORACLE (test infrastructure): turns the reference's shader files into C++.

Usage: python glsl_to_cpp.py <shader directory> <output directory>

Every *.sh and *.sc file of the reference's shader directory is written to
the output directory with the mechanical changes below and nothing else, so that
it compiles as C++ against oracle/ref_shim/shader_shim.h:

  * comments become blanks (newlines kept, so compiler messages keep the
    shader's own line numbers, give or take the line a private global's
    macro adds below);
  * floating-point literals get an `f` suffix: GLSL literals are single
    precision, C++ ones double, and a double literal would widen the
    arithmetic around it;
  * `out T name` and `inout T name` parameters become `T& name`;
  * a global declared `static` (a shader's private, per-invocation global,
    such as bvh.sh's g_bvhThread) becomes one slot per lane of the running
    worker (`static thread_local T name_lanes[kMaxLanes]` and a macro that
    indexes it by the running lane), since a group's lanes are coroutines of
    one worker thread;
  * GLSL evaluates a call's arguments left to right, C++ in no set order
    (g++ goes right to left): where one statement passes the results of
    several calls that update the same state through an `inout` parameter
    (`f(nextRandom(rng), nextRandom(rng))`), those calls are hoisted, in
    source order, into temporaries at the start of the statement (same
    line). Any other statement with more than one call to a function that
    has an `out`/`inout` parameter is refused, so nothing is reordered
    silently.

`#include <bgfx_compute.sh>`, `<bgfx_shader.sh>`, `<common.sh>` and
`"shaderlib.sh"` are dropped (the shim is included first and has the three
shaderlib helpers the shaders use), and so are the fragment shaders' bgfx
varying lines (`$input v_texcoord0`: the shim supplies v_texcoord0). The output goes to oracle/_ref/, which is never
committed: the shader sources stay where they are.
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

COMMENT = re.compile(r"//[^\n]*|/\*.*?\*/", re.S)
FLOAT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")
QUALIFIED = re.compile(r"\b(?:inout|out)\s+([A-Za-z_]\w*)\s+(_?[A-Za-z]\w*)")
PRIVATE_GLOBAL = re.compile(r"^static\s+(?!const\b)([A-Za-z_]\w*)\s+([A-Za-z_]\w*)\s*;", re.M)
IN_QUALIFIED = re.compile(r"([(,]\s*)in\s+([A-Za-z_]\w*\s+_?[A-Za-z]\w*)")
DROPPED = re.compile(r'^[ \t]*(?:#[ \t]*include[ \t]*(?:<bgfx_(?:compute|shader)\.sh>|<common\.sh>|"shaderlib\.sh")'
                     r'|\$(?:input|output)\b)[^\n]*$', re.M)


def blank(match: re.Match) -> str:
    return re.sub(r"[^\n]", " ", match.group(0))


OUT_FUNCTION = re.compile(r"\b[A-Za-z_]\w*\s+([A-Za-z_]\w*)\s*\([^;{)]*\b(?:inout|out)\s")
HOISTED = ("nextRandom",)


def argument_order(text: str, writers: set[str]) -> str:
    """Hoists the HOISTED calls out of a statement that passes several
    state-updating calls as arguments, in source order; refuses any other
    such statement. A call counts when it sits inside parentheses (an
    argument, or an operand within an argument): `selectLight(nextRandom(rng),
    pmf)` has one, `gridJitter(p, n, s, nextRandom(rng), nextRandom(rng))`
    two."""
    lines = text.split("\n")
    for i, line in enumerate(lines):
        inner = []
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(", line):
            depth = line[:m.start()].count("(") - line[:m.start()].count(")")
            if m.group(1) in writers and depth > 0:
                inner.append(m.group(1))
        if len(inner) < 2:
            continue
        if set(inner) - set(HOISTED) or not line.rstrip().endswith(";"):
            raise SystemExit(f"line {i + 1}: several calls with out/inout parameters in one statement: {line.strip()}")
        hoisted = []
        pattern = re.compile(r"\b(" + "|".join(HOISTED) + r")\s*\(([^()]*)\)")

        def replace(m, hoisted=hoisted):
            name = f"_ordered{len(hoisted)}"
            hoisted.append(f"float {name} = {m.group(1)}({m.group(2)});")
            return name
        body = pattern.sub(replace, line)
        indent = body[:len(body) - len(body.lstrip())]
        lines[i] = indent + " ".join(hoisted) + " " + body.lstrip()
    return "\n".join(lines)


def translate(text: str, writers: set[str]) -> str:
    """One shader file as C++; writers: the functions (of every shader file)
    that have an out or inout parameter."""
    text = COMMENT.sub(blank, text)
    text = DROPPED.sub("", text)
    text = argument_order(text, writers)
    text = FLOAT.sub(lambda m: m.group(1) + "f", text)
    text = QUALIFIED.sub(lambda m: f"{m.group(1)}& {m.group(2)}", text)
    text = IN_QUALIFIED.sub(lambda m: m.group(1) + m.group(2), text)
    text = PRIVATE_GLOBAL.sub(lambda m: f"static thread_local {m.group(1)} {m.group(2)}_lanes[refsh::kMaxLanes]; "
                              f"\n#define {m.group(2)} {m.group(2)}_lanes[refsh::t_lane]", text)
    return text


def main() -> None:
    source, target = Path(sys.argv[1]), Path(sys.argv[2])
    target.mkdir(parents=True, exist_ok=True)
    paths = sorted(list(source.glob("*.sh")) + list(source.glob("*.sc")))
    texts = {path: COMMENT.sub(blank, path.read_text()) for path in paths}
    writers = set()
    for text in texts.values():
        writers |= set(OUT_FUNCTION.findall(text))
    for path, text in texts.items():
        (target / path.name).write_text(translate(text, writers))


if __name__ == "__main__":
    main()
