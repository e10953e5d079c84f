#!/usr/bin/env python3
"""Generate tests/golden/sprp_vectors.txt: strong-PRP verdicts of the
reference's own strong_prp (src/common/PrimeQ_x86.h:143-182), computed by
oracle/_ref/ref_primeq (built from the reference sources by
oracle/build_ref.sh).  Test infrastructure.

Cases (seeded): small odd N, base-2 strong pseudoprimes, Carmichael numbers,
random odd N in [2^40, 2^62), primes and composites just below 2^62,
semiprimes of two ~31-bit primes, the terms of the golden APs and their
neighbours, and the 9 validation bases on a subset.  Each line: N a verdict.
"""
import os
import random
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TOOL = os.path.join(ROOT, "oracle", "_ref", "ref_primeq")
PRIM23 = 223092870


def sprp(a, n):
    d, t = n - 1, 0
    while d % 2 == 0:
        d //= 2
        t += 1
    x = pow(a, d, n)
    if x in (1, n - 1):
        return True
    for _ in range(t - 1):
        x = x * x % n
        if x == n - 1:
            return True
    return False


def is_prime(n):
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    return all(sprp(a, n) for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37))


def main():
    rng = random.Random(2626)
    cases = []
    cases += [(n, 2) for n in range(3, 400, 2)]
    psp = [n for n in range(3, 1 << 20, 2) if not is_prime(n) and sprp(2, n)][:40]
    cases += [(n, 2) for n in psp]
    cases += [(n, 2) for n in (561, 1105, 1729, 2465, 2821, 6601, 8911, 10585, 15841, 29341,
                               41041, 46657, 52633, 62745, 63973, 75361)]
    for _ in range(600):
        cases.append((rng.randrange(1 << 40, 1 << 62) | 1, 2))
    top = (1 << 62) - 1
    n = top
    got = 0
    while got < 60:
        if is_prime(n):
            cases.append((n, 2))
            got += 1
        elif got % 3 == 0:
            cases.append((n, 2))
        n -= 2
    small_primes = [p for p in range(1 << 30, (1 << 30) + 5000) if is_prime(p)]
    for _ in range(80):
        p, q = rng.sample(small_primes, 2)
        cases.append((p * q, 2))
    for first, k, K in ((6171054912832631, 25, 366384), (136926916457315893, 26, 44121555),
                        (161004359399459161, 26, 47715109)):
        for j in range(-2, k + 2):
            v = first + j * K * PRIM23
            if 0 < v < (1 << 62):
                cases.append((v, 2))
                if j in (0, k - 1):
                    for a in (3, 5, 7, 11, 13, 17, 19, 23):
                        cases.append((v, a))
    for _ in range(100):
        v = rng.randrange(1 << 40, 1 << 62) | 1
        cases.append((v, rng.choice((3, 5, 7, 11, 13, 17, 19, 23))))
    inp = "".join(f"{n} {a}\n" for n, a in cases)
    out = subprocess.run([TOOL], input=inp, capture_output=True, text=True, check=True).stdout
    lines = out.strip().splitlines()
    assert len(lines) == len(cases)
    for ln, (n, a) in zip(lines, cases):
        nn, aa, v = map(int, ln.split())
        assert (nn, aa) == (n, a)
        assert v == int(sprp(a, n)), (n, a, v)
    with open(os.path.join(HERE, "sprp_vectors.txt"), "w") as f:
        f.write("# N a verdict  -- reference strong_prp via oracle/_ref/ref_primeq\n")
        f.write("\n".join(lines) + "\n")
    print(len(lines), "vectors")


if __name__ == "__main__":
    main()
