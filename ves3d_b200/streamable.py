"""The reference's Streamable ASCII interchange format (include/Streamable.h:47-98), so that
surfaces and fields move between Ves3D checkpoints and this library:

    ARRAY     src/Array.cc:107-165      version, name, size, data
    SCALARS   src/Scalars.cc:220-285    version, nsubs, shorder, gridx, gridy, stride, ARRAY
    VECTORS   src/Vectors.cc:86-130     version, CoordinateOrder, SCALARS
    SURFACE   src/Surface.cc:608-680    version, name, orders and filter settings, VECTORS

Writers format numbers as the reference's checkpoints do (std::scientific with 16 digits,
src/Monitor.cc:72), which round-trips FP64 exactly. Readers take whitespace-separated
tokens as the reference's operator>> does and accept its version forms: a version with a
trailing "+" token, and the pre-591 layout with a "name:" key in the VECTORS and SCALARS
headers. Fields are numpy arrays in the reference's layout: a VECTORS block of n vectors at
order p holds [n][3][(p+1) 2p] (AxisMajor) or point-major data as its CoordinateOrder says.
"""
import numpy as np

VERSION = 1000  # any version above 590 selects the current header layout


def _num(x):
    return "%.16e" % x


# ---- writers --------------------------------------------------------------------------
def pack_array(name, data, version=VERSION):
    data = np.asarray(data, dtype=np.float64).reshape(-1)
    return ("ARRAY\n" f"version: {version}\n" f"name: {name}\n" f"size: {data.size}\n"
            "data: " + " ".join(_num(v) for v in data) + "\n/ARRAY\n")


def pack_scalars(name, data, p, n_subs, version=VERSION):
    """A Scalars (or the scalar part of a Vectors: n_subs = number of vectors, data of
    3 (p+1) 2p values per vector)."""
    stride = (p + 1) * 2 * p
    return ("SCALARS\n" f"version: {version}\n" f"nsubs: {n_subs}\n" f"shorder: {p}\n" f"gridx: {p + 1}\n"
            f"gridy: {2 * p}\n" f"stride: {stride}\n" + pack_array(name, data, version) + "/SCALARS\n")


def pack_vectors(name, data, p, n_vec, order="AxisMajor", version=VERSION):
    if order not in ("AxisMajor", "PointMajor"):
        raise ValueError("CoordinateOrder must be AxisMajor or PointMajor")
    data = np.asarray(data, dtype=np.float64).reshape(-1)
    if data.size != n_vec * 3 * (p + 1) * 2 * p:
        raise ValueError("data size does not match n_vec vectors of order p")
    return ("VECTORS\n" f"version: {version}\n" f"CoordinateOrder: {order}\n"
            + pack_scalars(name, data, p, n_vec, version) + "/VECTORS\n")


def pack_surface(name, X, p, n_vec, diff_filter_freq=None, reparam_filter_freq=None, rep_exponent=4.0,
                 reparam_type="BoxReparam", resample_order=None, version=VERSION):
    """A Surface block (Surface::pack): the reference's defaults are diff and reparam filter
    frequencies 2p/3 and a resampling order of 2p (the upsampled order of its forces)."""
    f = 2 * p // 3 if diff_filter_freq is None else diff_filter_freq
    rf = 2 * p // 3 if reparam_filter_freq is None else reparam_filter_freq
    ro = 2 * p if resample_order is None else resample_order
    return ("SURFACE\n" f"version: {version}\n" f"name: {name}\n" f"sh_order: {p}\n" f"SHT_order: {p}\n"
            f"SHT_rep_order: {p}\n" f"SHT_rep_exponent: {rep_exponent:g}\n" f"SHT_resample_order: {ro}\n"
            f"diff_filter_freq: {f}\n" f"reparam_filter_freq: {rf}\n" f"reparam_type: {reparam_type}\n"
            + pack_vectors("position", X, p, n_vec, "AxisMajor", version) + "/SURFACE\n")


# ---- readers --------------------------------------------------------------------------
class Tokens:
    """Whitespace-separated tokens of a text, read in order (the reference's operator>>)."""

    def __init__(self, text):
        self.t = text.split()
        self.i = 0

    def next(self):
        if self.i >= len(self.t):
            raise ValueError("unexpected end of the stream")
        self.i += 1
        return self.t[self.i - 1]

    def expect(self, word):
        w = self.next()
        if w != word:
            raise ValueError(f"bad stream: expected {word!r}, found {w!r}")

    def seek(self, word):
        """Advance to the next occurrence of a block header."""
        while self.i < len(self.t) and self.t[self.i] != word:
            self.i += 1
        if self.i >= len(self.t):
            raise ValueError(f"no {word} block")


def _version(tok, old_name_key):
    """version: N [+] ; returns (version, the next key). Pre-591 headers carry a name."""
    key = tok.next()
    version = 0
    if key == "version:":
        version = int(tok.next())
        key = tok.next()
        if key == "+":
            version += 1
            key = tok.next()
    if old_name_key and version <= 590:
        if key != "name:":
            raise ValueError("bad stream: expected 'name:'")
        tok.next()
        key = tok.next()
    return version, key


def unpack_array(tok):
    tok.expect("ARRAY")
    _, key = _version(tok, False)
    if key != "name:":
        raise ValueError("bad stream: expected 'name:'")
    name = tok.next()
    tok.expect("size:")
    n = int(tok.next())
    tok.expect("data:")
    data = np.array([float(tok.next()) for _ in range(n)], dtype=np.float64)
    tok.expect("/ARRAY")
    return name, data


def unpack_scalars(tok):
    """-> dict(name, data, p, n_subs, gridx, gridy, stride)."""
    tok.expect("SCALARS")
    _, key = _version(tok, True)
    if key != "nsubs:":
        raise ValueError("bad stream: expected 'nsubs:'")
    n_subs = int(tok.next())
    vals = {}
    for k in ("shorder:", "gridx:", "gridy:", "stride:"):
        tok.expect(k)
        vals[k] = int(tok.next())
    name, data = unpack_array(tok)
    tok.expect("/SCALARS")
    return dict(name=name, data=data, p=vals["shorder:"], n_subs=n_subs, gridx=vals["gridx:"], gridy=vals["gridy:"],
                stride=vals["stride:"])


def unpack_vectors(tok):
    """-> dict(name, data, p, n_vec, order, ...)."""
    tok.expect("VECTORS")
    _, key = _version(tok, True)
    if key != "CoordinateOrder:":
        raise ValueError("bad stream: expected 'CoordinateOrder:'")
    order = tok.next()
    sc = unpack_scalars(tok)
    tok.expect("/VECTORS")
    sc["order"] = order
    sc["n_vec"] = sc.pop("n_subs")
    return sc


def unpack_surface(tok):
    """-> dict(name, p, settings, X (AxisMajor [n][3][ng]), n_vec)."""
    tok.expect("SURFACE")
    _, key = _version(tok, False)
    if key != "name:":
        raise ValueError("bad stream: expected 'name:'")
    name = tok.next()
    settings = {}
    for k in ("sh_order:", "SHT_order:", "SHT_rep_order:", "SHT_rep_exponent:", "SHT_resample_order:",
              "diff_filter_freq:", "reparam_filter_freq:", "reparam_type:"):
        tok.expect(k)
        settings[k[:-1]] = tok.next()
    vec = unpack_vectors(tok)
    tok.expect("/SURFACE")
    X = vec["data"]
    if vec["order"].startswith("Poin"):  # point-major -> AxisMajor per vector
        ng = vec["stride"]
        X = X.reshape(vec["n_vec"], ng, 3).transpose(0, 2, 1).reshape(-1)
    return dict(name=name, p=int(settings["sh_order"]), settings=settings, X=X, n_vec=vec["n_vec"])


def read_surfaces(text):
    """Every SURFACE block of a text (a Ves3D checkpoint holds the parameters first, then
    the evolving state with its surface): list of unpack_surface results."""
    tok = Tokens(text)
    out = []
    while True:
        try:
            tok.seek("SURFACE")
        except ValueError:
            return out
        out.append(unpack_surface(tok))
