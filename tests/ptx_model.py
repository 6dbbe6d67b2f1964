"""A CPU model of the inline-PTX subset used by the Goldilocks arithmetic in
era-boojum-cuda_b200/csrc/gl.cuh.

`asm_blocks(path)` pulls every `asm("...")` block out of the header, keyed by
the enclosing function and its position inside it; `run(block, inputs)` executes
the block's instructions on Python integers with PTX semantics (32-bit
registers, one carry flag written by `.cc` forms and read by `addc`/`subc`/
`madc`, 64-bit packs and unpacks) and returns the output operands.  The tests
drive each block with the operands the C++ around it computes and compare with
exact arithmetic mod p, so the carry chains are checked without a GPU.
"""
from __future__ import annotations

import re

M32 = (1 << 32) - 1
M64 = (1 << 64) - 1

_FUNC = re.compile(r"__device__\s+__forceinline__\s+[\w:<>]+\s+(\w+)\s*\(")
_ASM = re.compile(r"asm\s*\(")


def _literal_text(body: str) -> str:
    """Concatenate the C string literals of an asm template (stops at the first ':')."""
    out, i = [], 0
    while i < len(body):
        ch = body[i]
        if ch == '"':
            j = i + 1
            buf = []
            while body[j] != '"':
                if body[j] == "\\":
                    nxt = body[j + 1]
                    buf.append({"n": "\n", "t": "\t", '"': '"', "\\": "\\"}[nxt])
                    j += 2
                else:
                    buf.append(body[j])
                    j += 1
            out.append("".join(buf))
            i = j + 1
        elif ch == ":":
            break
        elif body.startswith("//", i):
            i = body.index("\n", i)
        else:
            i += 1
    return "".join(out)


def asm_blocks(path: str) -> dict[tuple[str, int], str]:
    """{(function name, k-th asm block in it): template text}."""
    src = open(path).read()
    funcs = [(m.start(), m.group(1)) for m in _FUNC.finditer(src)]
    blocks: dict[tuple[str, int], str] = {}
    for m in _ASM.finditer(src):
        owner = None
        for start, name in funcs:
            if start < m.start():
                owner = name
        k = sum(1 for key in blocks if key[0] == owner)
        blocks[(owner, k)] = _literal_text(src[m.end():])
    return blocks


def _imm(tok: str):
    tok = tok.strip()
    if re.fullmatch(r"0x[0-9a-fA-F]+|\d+", tok):
        return int(tok, 0)
    if re.fullmatch(r"-\d+", tok):
        return int(tok) & M32
    return None


def compile_block(block: str) -> list[tuple[str, list[str]]]:
    """Split a template into (opcode, operand tokens), dropping the scope braces and .reg lines."""
    prog = []
    for raw in block.split(";"):
        line = re.sub(r"^\{\s*", "", raw.strip())  # statements start with an opcode, never a pack
        if not line or line == "}" or line.startswith(".reg"):
            continue
        op, _, rest = line.partition(" ")
        prog.append((op, [a.strip() for a in re.split(r",(?![^{]*\})", rest)]))
    return prog


def run(block, inputs: list[int], outputs: int = 1):
    """Execute a template (text or compile_block output); inputs bind %<outputs>, %<outputs+1>, ...
    Returns %0, or the tuple (%0, ..., %<outputs-1>)."""
    prog = compile_block(block) if isinstance(block, str) else block
    regs: dict[str, int] = {}
    for i, v in enumerate(inputs, start=outputs):
        regs[f"%{i}"] = v
    cf = 0

    def val(tok):
        v = _imm(tok)
        return v if v is not None else regs[tok]

    for op, args in prog:
        if op == "mov.b64":
            dst, src = args
            if dst.startswith("{"):
                lo, hi = [t.strip() for t in dst.strip("{} ").split(",")]
                x = val(src)
                regs[lo], regs[hi] = x & M32, (x >> 32) & M32
            elif src.startswith("{"):
                lo, hi = [t.strip() for t in src.strip("{} ").split(",")]
                regs[dst] = (val(lo) & M32) | ((val(hi) & M32) << 32)
            else:
                regs[dst] = val(src) & M64
            continue
        if op == "mov.u32":
            regs[args[0]] = val(args[1]) & M32
            continue
        d = args[0]
        a = [val(t) for t in args[1:]]
        parts = op.split(".")
        base, flags = parts[0], parts[1:]
        cc = "cc" in flags
        if base in ("add", "addc"):
            r = a[0] + a[1] + (cf if base == "addc" else 0)
            if cc:
                cf = r >> 32
            regs[d] = r & M32
        elif base in ("sub", "subc"):
            r = a[0] - a[1] - (cf if base == "subc" else 0)
            if cc:
                cf = 1 if r < 0 else 0
            regs[d] = r & M32
        elif base == "neg":
            regs[d] = (-a[0]) & M32
        elif base == "not":
            regs[d] = (~a[0]) & M32
        elif base == "mul":
            prod = (a[0] & M32) * (a[1] & M32)
            if "wide" in flags:
                regs[d] = prod & M64
            else:
                regs[d] = (prod >> 32) & M32 if "hi" in flags else prod & M32
        elif base in ("mad", "madc"):
            prod = (a[0] & M32) * (a[1] & M32)
            if "wide" in flags:
                regs[d] = (prod + a[2]) & M64
                continue
            part = (prod >> 32) & M32 if "hi" in flags else prod & M32
            r = part + (a[2] & M32) + (cf if base == "madc" else 0)
            if cc:
                cf = r >> 32
            regs[d] = r & M32
        elif base == "setp":
            regs[d] = {"ne": a[0] != a[1], "eq": a[0] == a[1]}[flags[0]]
        elif base == "selp":
            regs[d] = a[0] if a[2] else a[1]
        else:
            raise NotImplementedError(op)
    if outputs == 1:
        return regs["%0"]
    return tuple(regs[f"%{i}"] for i in range(outputs))
