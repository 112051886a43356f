"""Result writers in the reference's formats (host side, FP64 copies of the state).

write_vtk   <- QDsim.ouputVTK  (src/QDsim.py:1142-1289): legacy VTK ASCII unstructured
             grid, 17 cell fields in the reference's order and number formats
             (byte-identical output for the same state).
write_txt   <- QDsim.outputtxt (src/QDsim.py:1301-1368): slip-rate and traction maps
             interpolated (cubic) on a 500 x 300 grid of the x-z plane, into out_txt/.
StateLog    <- the state.txt header and per-step lines of src/main.py:83-99,177.
"""
import os
from datetime import datetime

import numpy as np

VTK_FIELDS = [("Normal_[MPa]", "Tno", "%f"), ("Shear_[MPa]", "Tt", "%f"), ("Shear_1[MPa]", "Tt1o", "%f"),
              ("Shear_2[MPa]", "Tt2o", "%f"), ("rake[Degree]", "rake_deg", "%f"), ("state", "state", "%f"),
              ("Slipv[m/s]", "slipv", "%.40f"), ("Slipv1[m/s]", "slipv1", "%.40f"),
              ("Slipv2[m/s]", "slipv2", "%.40f"), ("a", "a", "%f"), ("b", "b", "%f"), ("a-b", "a_b", "%f"),
              ("dc", "dc", "%.10f"), ("fric", "fric", "%f"), ("slip", "slip", "%.20f"), ("slip1", "slip1", "%.20f"),
              ("slip2", "slip2", "%.20f"), ("slip_plate", "slipvC", "%.15f")]


def _join(fmt, arr):
    return "".join((fmt + " ") % v for v in np.asarray(arr, dtype=np.float64).tolist())


def vtk_text(sim):
    n_node = sim.nodelst.shape[0]
    n_ele = sim.elelst.shape[0]
    parts = ["# vtk DataFile Version 3.0\n", "test\n", "ASCII\n", "DATASET  UNSTRUCTURED_GRID\n",
             "POINTS " + str(n_node) + " float\n"]
    parts += ["%f %f %f\n" % (p[0], p[1], p[2]) for p in np.asarray(sim.nodelst, dtype=np.float64).tolist()]
    parts.append("CELLS " + str(n_ele) + " " + str(n_ele * 4) + "\n")
    parts += ["3 %d %d %d\n" % (t[0] - 1, t[1] - 1, t[2] - 1) for t in np.asarray(sim.elelst).tolist()]
    parts.append("CELL_TYPES " + str(n_ele) + "\n")
    parts.append("5 " * n_ele)
    parts.append("\n")
    parts.append("CELL_DATA %d " % n_ele)
    values = dict(rake_deg=np.asarray(sim.rake) * 180. / np.pi, a_b=np.asarray(sim.a) - np.asarray(sim.b))
    for label, attr, fmt in VTK_FIELDS:
        v = values[attr] if attr in values else getattr(sim, attr)
        parts.append("SCALARS " + label + " float\nLOOKUP_TABLE default\n")
        parts.append(_join(fmt, v))
        parts.append("\n")
    return "".join(parts)


def write_vtk(sim, fname):
    with open(fname, "w") as f:
        f.write(vtk_text(sim))


def write_txt(sim, fname, directory="out_txt"):
    from scipy.interpolate import griddata
    os.makedirs(directory, exist_ok=True)
    xg = sim.xg
    xmin, xmax = np.min(xg[:, 0]), np.max(xg[:, 0])
    zmin, zmax = np.min(xg[:, 2]), np.max(xg[:, 2])
    X1 = np.linspace(xmin + sim.maxsize, xmax - sim.maxsize, 500)
    Y1 = np.linspace(zmin + sim.maxsize, zmax - sim.maxsize, 300)
    Xg, Yg = np.meshgrid(X1, Y1)
    mesh1 = np.column_stack((Xg.flatten(), Yg.flatten()))

    def grid(fn, arr, fmt):
        with open(os.path.join(directory, fn), "w") as f:
            for row in arr:
                f.write("".join((fmt + " ") % v for v in row.tolist()))
                f.write("\n")
    grid("X_grid.txt", Xg, "%f")
    grid("Y_grid.txt", Yg, "%f")
    for suffix, values in (("slipv", sim.slipv), ("slipv1", sim.slipv1), ("slipv2", sim.slipv2), ("Traction", sim.Tt)):
        m = griddata(xg[:, [0, 2]], values, mesh1, method="cubic").reshape((Y1.shape[0], X1.shape[0]))
        grid(fname + suffix + ".txt", m, "%.5f")


class StateLog:
    """state.txt of the reference driver: header, one line per step, timing footer."""

    def __init__(self, path, sim, fnamegeo, fnamePara, nodes, tris):
        self.f = open(path, "w")
        f = self.f
        f.write("Program start time: %s\n" % str(datetime.now()))
        f.write("Input msh geometry file:%s\n" % fnamegeo)
        f.write("Input parameter file:%s\n" % fnamePara)
        f.write("Number of Node:%d\n" % nodes.shape[0])
        f.write("Number of Element:%d\n" % tris.shape[0])
        f.write("Cs:%f\n" % sim.Cs)
        f.write("First Lamé constants:%f\n" % sim.lambda_)
        f.write("Shear Modulus:%f\n" % sim.mu)
        f.write("Youngs Modulus:%f\n" % sim.YoungsM)
        f.write("Poissons ratio:%f\n" % sim.possonratio)
        f.write("maximum element size:%f\n" % sim.maxsize)
        f.write("average elesize:%f\n" % sim.ave_elesize)
        f.write("Critical nucleation size:%f\n" % sim.hRA)
        f.write("Cohesive zone::%f\n" % sim.A0)
        f.write("iteration time_step(s) maximum_slip_rate(m/s) time(s) time(h)\n")

    def step(self, i, dt, maxv1, maxv2, t):
        self.f.write("%d %f %f %.16e %f %f\n" % (i, dt, maxv1, maxv2, t, t / 3600.0 / 24.0))

    def close(self, seconds):
        self.f.write("Program end time: %s\n" % str(datetime.now()))
        self.f.write("Time taken: %.2f seconds\n" % seconds)
        self.f.close()
