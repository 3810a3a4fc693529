"""Writes tests/golden/kat.json: the known-answer data of the reference's tests.

* The 3x3 systems of linalg/GMResTest.java:22-39, 83-91, 111-123 and
  linalg/BiCGStabTest.java:22-39, 79-125 with b = (3, 4, 5); their exact
  solutions are computed here in rational arithmetic (Cramer's rule with
  fractions), independently of any solver under test.
* The identity systems of GMResTest.testIdentity (15x15, b = 1..15).
* java.util.Random: first nextDouble() values of new Random(42) and
  new Random(0) as documented for the JDK's 48-bit LCG (0.7275636800328681
  and 0.730967787376657), which pin the generator port used for the seeded
  fixtures of linalg/SparseMvMulTest.java:12-113.

Run:  python tests/golden/make_golden.py
"""
import json
import os
from fractions import Fraction

HERE = os.path.dirname(os.path.abspath(__file__))


def det3(m):
    return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1])
            - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0])
            + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]))


def cramer(a, b):
    A = [[Fraction(v) for v in row] for row in a]
    B = [Fraction(v) for v in b]
    d = det3(A)
    out = []
    for j in range(3):
        M = [row[:] for row in A]
        for i in range(3):
            M[i][j] = B[i]
        out.append(det3(M) / d)
    return out


def main():
    b = [3, 4, 5]
    systems = {
        "symm": [[0, 1, 2], [1, 0, 3], [2, 3, 0]],
        "nonsymm": [[3, 1, 7], [2, 0, 3], [2, 3, 0]],
        "good_nonsymm": [[3, 1, 7], [2, 4, 3], [2, 3, 7]],
    }
    kat = {}
    for name, a in systems.items():
        x = cramer(a, b)
        kat[name] = {"A": a, "b": b, "x": [float(v) for v in x], "x_exact": [str(v) for v in x]}
    kat["identity15"] = {"n": 15, "b": list(range(1, 16))}
    data = {
        "systems": kat,
        "java_random_first_double": {"42": 0.7275636800328681, "0": 0.730967787376657},
        "source": "linalg/GMResTest.java, linalg/BiCGStabTest.java, java.util.Random specification",
    }
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
