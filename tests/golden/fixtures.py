"""Access to the committed golden fixtures (see make_fixtures.py)."""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
INPUTS = os.path.join(HERE, "shipped_inputs.npz")
OUTPUTS = os.path.join(HERE, "reference_outputs.npz")


def key(name):
    return name.replace("/", "__").replace(".txt", "").replace(".csv", "")


def fmt6(v):
    """integer micro-degrees -> the six-decimal text the shipped files use"""
    s = "-" if v < 0 else ""
    v = abs(int(v))
    return "%s%d.%06d" % (s, v // 1000000, v % 1000000)


class Inputs:
    def __init__(self, path=INPUTS):
        self.z = np.load(path)

    def polygons(self):
        return sorted({k[5:-6] for k in self.z.files if k.startswith("poly_") and k.endswith("_heads")})

    def rings_micro(self, name):
        k = key(name)
        heads = self.z["poly_%s_heads" % k]
        return heads, [self.z["poly_%s_ring%d" % (k, i)] for i in range(len(heads))]

    def rings_deg(self, name):
        """Rings as float64 degrees without the closing vertex, parsed like sscanf would."""
        heads, rings = self.rings_micro(name)
        return [np.array([[float(fmt6(a)), float(fmt6(b))] for a, b in r[:-1]]) for r in rings]

    def polygon_text(self, name):
        heads, rings = self.rings_micro(name)
        lines = ["POLYGON 1 %d" % (len(rings) - 1)]
        for (a, b), r in zip(heads, rings):
            lines.append("%d %d" % (a, b))
            lines.extend("%s %s" % (fmt6(x), fmt6(y)) for x, y in r)
        return "\n".join(lines) + "\n"

    def polygon_file(self, name, directory):
        path = os.path.join(directory, key(name) + ".txt")
        with open(path, "w") as f:
            f.write(self.polygon_text(name))
        return path

    def query(self, name):
        m = self.z["query_" + key(name)]
        return np.array([[float(fmt6(a)), float(fmt6(b))] for a, b in m])

    def query_file(self, name, directory):
        m = self.z["query_" + key(name)]
        path = os.path.join(directory, key(name) + ".csv")
        with open(path, "w") as f:
            f.write("".join("%s,%s\n" % (fmt6(a), fmt6(b)) for a, b in m))
        return path


class Outputs:
    def __init__(self, path=OUTPUTS):
        self.z = np.load(path)

    def get(self, what, name):
        return self.z["%s_%s" % (what, key(name))]
