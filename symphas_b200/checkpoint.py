"""SymPhas's checkpoint files for device-resident fields.

SymPhas checkpoints a field as text (symphas::io::gp::save_grid,
io/src/writegp.cpp:780-806, header print_gp_header :425-465): a header line

    <dim> <n_x> [<n_y> [<n_z>]] <left_x> <right_x> [...] <index> @

(counts, then the domain end points of each axis, "%d " and "%lf %lf ", the
solution index and "@" for a grid without a sub-domain), then the values
"%.10E " with x fastest and a newline after each x-row.  The files live in
<dir>/checkpoint/ named data<id> (one file holding every save) or
data<id>_<index> (one per save) (io/inc/io.h:184-188).  The reader follows
symphas::io::gp::read_header (io/src/readgp.cpp:46-130).

save() downloads the interior of a field and writes that format; load() reads
it back and uploads it (the halo is refreshed on upload).  Values keep the
ten decimal digits of the format, as SymPhas's own checkpoints do.
"""
import os

import numpy as np


def checkpoint_path(out_dir, field_id, index=None):
    """<out_dir>/checkpoint/data<id>[_<index>], SymPhas's checkpoint names."""
    name = "data%d" % field_id if index is None else "data%d_%d" % (field_id, index)
    return os.path.join(out_dir, "checkpoint", name)


def header(dims, h, index, left=None):
    """The header line for a grid of `dims` (x first) points of spacing h."""
    dims = [int(v) for v in dims]
    left = [0.0] * len(dims) if left is None else list(left)
    s = "%d " % len(dims)
    s += "".join("%d " % n for n in dims)
    s += "".join("%f %f " % (l, l + (n - 1) * h) for n, l in zip(dims, left))
    return s + "%d @\n" % index


def format_values(values):
    """The data block: '%.10E ' per value, x fastest, newline per x-row."""
    a = np.asarray(values, dtype=np.float64)
    rows = a.reshape(-1, a.shape[-1])
    return "".join("".join("%.10E " % v for v in row) + "\n" for row in rows)


def write(f, values, h, index, left=None):
    a = np.asarray(values)
    f.write(header(tuple(reversed(a.shape)), h, index, left))
    f.write(format_values(a))


def read(f):
    """Read one save: returns (index, dims (x first), (left, right) per axis,
    values shaped (z, y, x) / (y, x))."""
    tok = f.read().split()
    dim = int(tok[0])
    dims = [int(t) for t in tok[1:1 + dim]]
    p = 1 + dim
    ends = [(float(tok[p + 2 * a]), float(tok[p + 2 * a + 1])) for a in range(dim)]
    p += 2 * dim
    index = int(tok[p])
    p += 1
    if tok[p] != "@":  # a sub-domain: its dimension and end points follow
        p += 1 + 2 * int(tok[p])
    else:
        p += 1
    count = int(np.prod(dims))
    values = np.array([float(t) for t in tok[p:p + count]], dtype=np.float64)
    if values.size != count:
        raise ValueError("checkpoint holds %d values, expected %d" % (values.size, count))
    return index, dims, ends, values.reshape(tuple(reversed(dims)))


def save(model, out_dir, index, field=0, inst=0, field_id=None, per_index=True):
    """Write field `field` of instance `inst` of a model (any Model of this
    package) as SymPhas's checkpoint; returns the path."""
    path = checkpoint_path(out_dir, field if field_id is None else field_id,
                           index if per_index else None)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w" if per_index else "a") as f:
        write(f, model.get_field(field, inst), model.desc.h, index)
    return path


def load(model, path, field=0, inst=0):
    """Read a SymPhas checkpoint into field `field` of instance `inst`;
    returns the solution index it holds."""
    with open(path) as f:
        index, dims, _, values = read(f)
    model.set_field(field, values.astype(model.np_dtype), inst=inst)
    return index
