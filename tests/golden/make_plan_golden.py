"""Regenerate tests/golden/ref_plans.jsonl from the reference's own planner.

Runs oracle/_ref/ref_plan_dump (built by `make -C oracle ref` from the reference
sources: src/query/*.h and bliss 0.73) over every preset pattern (-p 0..18),
every clique size (-kc 3..7), every graphlet set (-km 3..5) and a fixed set of
seeded random connected patterns of 3..7 vertices with edge probability 0.5, and
stores each plan as one JSON line.  The random patterns' adjacency is stored next
to the plan so the product planner can be fed the same input.

    python tests/golden/make_plan_golden.py
"""
import json
import os
import random
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DUMP = os.path.join(HERE, "..", "..", "oracle", "_ref", "ref_plan_dump")


def random_patterns(count, seed):
    rng = random.Random(seed)
    out = []
    while len(out) < count:
        n = rng.randint(3, 7)
        bits = [[0] * n for _ in range(n)]
        for i in range(n):
            for j in range(i + 1, n):
                if rng.random() < 0.5:
                    bits[i][j] = bits[j][i] = 1
        # connectivity
        seen = {0}
        stack = [0]
        while stack:
            x = stack.pop()
            for y in range(n):
                if bits[x][y] and y not in seen:
                    seen.add(y)
                    stack.append(y)
        if len(seen) == n:
            out.append((n, "".join(str(bits[i][j]) for i in range(n) for j in range(n))))
    return out


def run(args, stdin=None):
    res = subprocess.run([DUMP] + args, input=stdin, capture_output=True, text=True, check=True)
    return [json.loads(line) for line in res.stdout.splitlines() if line.startswith("{")]


def main():
    if not os.path.exists(DUMP):
        sys.exit("build oracle/_ref first: make -C oracle ref")
    rows = []
    for p in range(19):
        rows += run(["-p", str(p)])
    for k in range(3, 8):
        rows += run(["-kc", str(k)])
    for k in range(3, 6):
        rows += run(["-km", str(k)])
    pats = random_patterns(400, seed=20240607)
    rand = run(["-stdin"], stdin="".join(f"{n} {b}\n" for n, b in pats))
    for (n, b), row in zip(pats, rand):
        row["input_n"] = n
        row["input_bits"] = b
    rows += rand
    with open(os.path.join(HERE, "ref_plans.jsonl"), "w") as f:
        for r in rows:
            f.write(json.dumps(r, separators=(",", ":")) + "\n")
    print(f"wrote {len(rows)} plans")


if __name__ == "__main__":
    main()
