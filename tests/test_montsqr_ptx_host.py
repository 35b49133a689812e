"""The prover's Montgomery squares (montsqr<3>, montsqr<4> in csrc/prove.cu)
are hand-written PTX carry chains.  This host test reads those asm blocks
from the source, runs them instruction by instruction on 32-bit words with a
carry flag, and compares the result with a^2 R^-1 mod n in big-integer
arithmetic: random and edge operands, moduli of every bit length the
specialisations serve.  An instruction without a carry-out whose sum does not
fit 32 bits fails the test (a carry that the chain would drop)."""
import os
import random
import re

import pytest

SRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "cunningham-chain-search_b200", "csrc", "prove.cu")
M32 = (1 << 32) - 1


def _instructions(block):
    """PTX instructions of the string literals in a block of C source."""
    text = "".join(re.findall(r'"((?:[^"\\]|\\.)*)"', block))
    text = text.replace("\\n", "\n").replace("\\t", "")
    out = []
    for line in text.split("\n"):
        line = line.split("//")[0].strip().rstrip(";")
        if not line:
            continue
        op, rest = line.split(None, 1)
        out.append((op, [x.strip() for x in rest.split(",")]))
    return out


def _operands(block):
    """C expressions of the asm operands, in %-number order."""
    return re.findall(r'"\+?r"\(([^)]*(?:\[[0-9]\])?)\)', block)


def _asm_blocks(text):
    """(instructions, operand expressions) of every asm(...) statement."""
    res = []
    for m in re.finditer(r"asm\(", text):
        depth, i = 0, m.end() - 1
        while True:
            c = text[i]
            depth += c == "("
            depth -= c == ")"
            if depth == 0:
                break
            i += 1
        body = text[m.end():i]
        strings, _, ops = body.partition(":")
        res.append((_instructions(strings), _operands(":" + ops)))
    return res


def _run(prog, env, names):
    cc = 0

    def val(x):
        if x.startswith("%"):
            return env[names[int(x[1:])]]
        return int(x, 0)

    for op, args in prog:
        base = op.split(".")
        d = names[int(args[0][1:])]
        src = [val(x) for x in args[1:]]
        setcc = base[-2] == "cc" if len(base) > 2 else False
        kind = base[0]
        if kind == "mul":
            assert base[1] == "lo"
            env[d] = (src[0] * src[1]) & M32
            continue
        if kind in ("mad", "madc"):
            p = src[0] * src[1]
            p = p & M32 if base[1] == "lo" else p >> 32
            s = p + src[2] + (cc if kind == "madc" else 0)
        elif kind in ("add", "addc"):
            s = src[0] + src[1] + (cc if kind == "addc" else 0)
        else:
            raise AssertionError(f"unexpected instruction {op}")
        env[d] = s & M32
        if setcc:
            cc = s >> 32
        else:
            assert s >> 32 == 0, f"carry dropped by {op} {args}"


def _montsqr_sim(NL):
    text = open(SRC).read()
    fn = re.search(r"void montsqr<%d>\(.*?\n}\n" % NL, text, re.S).group(0)
    mac = re.search(r"#define CCS_SQR_ROW%d\((.*?)\)(.*?)\n\n" % NL, text, re.S)
    mac_params = [x.strip() for x in mac.group(1).split(",")]
    (sq_prog, sq_ops), = _asm_blocks(fn)
    (row_prog, row_ops), = _asm_blocks(mac.group(2).replace("\\\n", "\n"))
    calls = re.findall(r"CCS_SQR_ROW%d\(([^)]*)\)" % NL, fn)
    assert len(calls) == NL

    def sq(a, n, ninv):
        env = {f"t{k}": 0 for k in range(2 * NL)}
        for i in range(NL):
            env[f"a[{i}]"] = (a >> (32 * i)) & M32
            env[f"n[{i}]"] = (n >> (32 * i)) & M32
        _run(sq_prog, env, sq_ops)
        assert sum(env[f"t{k}"] << (32 * k) for k in range(2 * NL)) == a * a
        p = 0
        for call in calls:
            regs = [x.strip() for x in call.split(",")]
            m = (env[regs[0]] * ninv) & M32
            local = dict(env)
            local.update({"p": p, "m": m, "q": 0})
            for par, reg in zip(mac_params, regs):
                local[par] = env[reg]
            _run(row_prog, local, row_ops)
            for par, reg in zip(mac_params, regs):
                env[reg] = local[par]
            assert env[regs[0]] == 0
            p = local["q"]
        res = sum(env[f"t{NL + k}"] << (32 * k) for k in range(NL)) + (p << (32 * NL))
        return res - n if res >= n else res
    return sq


@pytest.mark.parametrize("NL", [3, 4])
def test_montsqr_ptx_matches_bigint(NL):
    sq = _montsqr_sim(NL)
    R = 1 << (32 * NL)
    rng = random.Random(20261204 + NL)
    moduli = []
    for bits in range(32 * (NL - 1) + 1, 32 * NL + 1):
        for _ in range(3):
            moduli.append(rng.getrandbits(bits) | 1 | (1 << (bits - 1)))
    moduli += [R - 1, R - 3, (1 << (32 * (NL - 1))) + 1]
    checked = 0
    for n in moduli:
        ninv = (-pow(n, -1, 1 << 32)) & M32
        rinv = pow(R, -1, n)
        for a in [0, 1, 2, n - 1, n - 2, n // 2] + [rng.randrange(n) for _ in range(8)]:
            assert sq(a, n, ninv) == a * a * rinv % n, (NL, hex(n), hex(a))
            checked += 1
    assert checked > 1000
