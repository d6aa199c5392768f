"""Counter-based uniform draws shared by the workload definitions (splitmix64
finaliser over a seed-salted counter; the same function the native generators use)."""

MASK = (1 << 64) - 1


def mix64(seed, i):
    z = (seed * 0x9E3779B97F4A7C15 + i * 0xD1B54A32D192ED03 + 0x632BE59BD9B4E019) & MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def stream_uniform(seed, i):
    return (mix64(seed, i) >> 11) * (1.0 / 9007199254740992.0)
