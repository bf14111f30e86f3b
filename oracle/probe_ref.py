"""CPU restatement of the reference's probe interpolation (TEST
INFRASTRUCTURE ONLY): ProbeOutput::SetupInterpolation
(ProbeOutput.cpp:219-340) and ProbeOutput::InterpolateSolutionAtProbe
(636-673) with MathTools::trilinear_interpolation (local-coordinate form,
MathTools/trilinear_interpolation.h). ProbeOutput.cpp itself does not build
in the oracle (it needs PETSc viewers), so this file follows its lines,
including SpaceVariable3D::OutsidePhysicalDomainAndUnpopulated
(SpaceVariable.h:150-159), which tests j (not i) against NX on the x axis.
Operates on the ghosted host state (m2cg_download_state layout) with plain
IEEE double arithmetic in the reference's operation order."""


def ghosted_coords(centres, widths):
    """Cell centres with one ghost per side (x_0 - dx_0, x_{N-1} + dx_{N-1},
    SpaceOperator::PopulateGhostBoundaryCoordinates); index c + 1 for c in
    [-1, N]."""
    out = [float(centres[0]) - float(widths[0])]
    out += [float(x) for x in centres]
    out.append(float(centres[-1]) + float(widths[-1]))
    return out


def setup(points, coords, N):
    """(i, j, k), trilinear coordinates and valid-corner flags per point."""
    NX, NY, NZ = N

    def unpopulated(i, j, k):
        count = 0
        if i < 0 or j >= NX:
            count += 1
        if j < 0 or j >= NY:
            count += 1
        if k < 0 or k >= NZ:
            count += 1
        return count > 1

    res = []
    for p in points:
        ijk, xi = [], []
        for a in range(3):
            X = coords[a]
            if p[a] < X[0] or p[a] >= X[N[a] + 1]:
                raise ValueError("probe outside the ghosted mesh")
            for i in range(-2, N[a]):
                if p[a] < X[i + 2]:
                    ijk.append(i)
                    xi.append((p[a] - X[i + 1]) / (X[i + 2] - X[i + 1]))
                    break
        i, j, k = ijk
        valid = [not unpopulated(i, j, k), not unpopulated(i + 1, j, k), not unpopulated(i, j + 1, k),
                 not unpopulated(i + 1, j + 1, k), not unpopulated(i, j, k + 1), not unpopulated(i + 1, j, k + 1),
                 not unpopulated(i, j + 1, k + 1), not unpopulated(i + 1, j + 1, k + 1)]
        res.append((ijk, xi, valid))
    return res


def interpolate(V, setup_entry, comp):
    """Component comp of the ghosted state V [nz+2][ny+2][nx+2][5] at one probe."""
    (i, j, k), xi, valid = setup_entry
    at = lambda a, b, c: float(V[c + 1, b + 1, a + 1, comp])
    c = [at(i, j, k) if valid[0] else 0.0, at(i + 1, j, k) if valid[1] else 0.0,
         at(i, j + 1, k) if valid[2] else 0.0, at(i + 1, j + 1, k) if valid[3] else 0.0,
         at(i, j, k + 1) if valid[4] else 0.0, at(i + 1, j, k + 1) if valid[5] else 0.0,
         at(i, j + 1, k + 1) if valid[6] else 0.0, at(i + 1, j + 1, k + 1) if valid[7] else 0.0]
    nv = sum(valid)
    if nv < 8:
        avg = (c[0] + c[1] + c[2] + c[3] + c[4] + c[5] + c[6] + c[7]) / nv
        c = [c[q] if valid[q] else avg for q in range(8)]
    c000, c100, c010, c110, c001, c101, c011, c111 = c
    c00 = c000 * (1.0 - xi[0]) + c100 * xi[0]
    c01 = c001 * (1.0 - xi[0]) + c101 * xi[0]
    c10 = c010 * (1.0 - xi[0]) + c110 * xi[0]
    c11 = c011 * (1.0 - xi[0]) + c111 * xi[0]
    c0 = c00 * (1.0 - xi[1]) + c10 * xi[1]
    c1 = c01 * (1.0 - xi[1]) + c11 * xi[1]
    return c0 * (1.0 - xi[2]) + c1 * xi[2]
