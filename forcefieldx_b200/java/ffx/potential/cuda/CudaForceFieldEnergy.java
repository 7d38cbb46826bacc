// Drop-in ForceFieldEnergy for Force Field X whose van der Waals and AMOEBA PME terms run in
// libffxcuda.so on one B200, through the FFM binding FfxCuda.
//
// Not compiled in this repository: no JDK is installed on the build machine (closed: no JDK
// on this box).  The class follows OpenMMEnergy (modules/potential/src/main/java/ffx/
// potential/openmm/OpenMMEnergy.java:80-631), the reference's precedent for a platform
// subclass: the platform key selects it in ForceFieldEnergy.energyFactory
// (ForceFieldEnergy.java:1464-1510), and it overrides the same methods.  The CPU keeps the
// bonded terms: the constructor puts the parent in its FAST term state
// (ForceFieldEnergy.setEnergyTermState, ForceFieldEnergy.java:2034-2076), which turns off
// van der Waals, permanent multipoles and polarization there, and every evaluation adds the
// library's terms to the parent's.
package ffx.potential.cuda;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;
import static java.lang.foreign.ValueLayout.JAVA_LONG;

import ffx.crystal.Crystal;
import ffx.potential.ForceFieldEnergy;
import ffx.potential.MolecularAssembly;
import ffx.potential.Platform;
import ffx.potential.bonded.Atom;
import ffx.potential.nonbonded.ParticleMeshEwald;
import ffx.potential.nonbonded.VanDerWaals;
import ffx.potential.nonbonded.VanDerWaalsForm;
import ffx.potential.parameters.ForceField;
import ffx.potential.parameters.MultipoleType;
import ffx.potential.parameters.PolarizeType;
import ffx.potential.utils.EnergyException;
import java.lang.foreign.Arena;
import java.lang.foreign.MemoryLayout.PathElement;
import java.lang.foreign.MemorySegment;
import java.lang.invoke.VarHandle;
import java.util.ArrayList;
import java.util.HashMap;
import java.util.List;
import java.util.Map;
import java.util.logging.Logger;

/** ForceFieldEnergy with the vdW + PME terms on the GPU (libffxcuda.so). */
public class CudaForceFieldEnergy extends ForceFieldEnergy {

  private static final Logger logger = Logger.getLogger(CudaForceFieldEnergy.class.getName());

  private final Arena arena = Arena.ofShared();
  private final Atom[] atoms;
  private final int nAtoms;
  private final boolean gpuLambda;
  private MemorySegment handle = MemorySegment.NULL;
  private final MemorySegment xyz, grad, terms, counts, dEdL, d2EdL2, lambdaGrad, box3, angles3, systemStruct;
  private STATE termState = STATE.BOTH;

  /**
   * @param molecularAssembly the system (every atom active) in P1: a crystal's space-group mates
   *                          are expanded into the P1 cell first.
   * @param nThreads          threads of the parent's bonded terms.
   */
  public CudaForceFieldEnergy(MolecularAssembly molecularAssembly, int nThreads) {
    super(molecularAssembly, nThreads);
    atoms = molecularAssembly.getAtomArray();
    nAtoms = atoms.length;
    Crystal crystal = getCrystal();
    if (crystal.spaceGroup.getNumberOfSymOps() > 1) {
      throw new EnergyException(" libffxcuda takes a P1 cell (expand the space group's mates first)");
    }
    ForceField ff = molecularAssembly.getForceField();
    xyz = arena.allocate(JAVA_DOUBLE, 3L * nAtoms);
    grad = arena.allocate(JAVA_DOUBLE, 3L * nAtoms);
    lambdaGrad = arena.allocate(JAVA_DOUBLE, 3L * nAtoms);
    terms = arena.allocate(JAVA_DOUBLE, FfxCuda.N_TERMS);
    counts = arena.allocate(JAVA_LONG, FfxCuda.N_COUNTS);
    dEdL = arena.allocate(JAVA_DOUBLE);
    d2EdL2 = arena.allocate(JAVA_DOUBLE);
    box3 = arena.allocate(JAVA_DOUBLE, 3);
    angles3 = arena.allocate(JAVA_DOUBLE, 3);
    systemStruct = arena.allocate(FfxCuda.SYSTEM);
    fillSystem(systemStruct);
    MemorySegment params = arena.allocate(FfxCuda.PARAMS);
    fillParams(params, ff, crystal);
    MemorySegment out = arena.allocate(ADDRESS);
    int st = call(() -> (int) FfxCuda.CREATE.invokeExact(systemStruct, params, out));
    if (st != FfxCuda.OK) {
      throw new EnergyException(" ffxg_create: " + FfxCuda.lastError(MemorySegment.NULL) + " (status " + st + ")");
    }
    handle = out.get(ADDRESS, 0);
    gpuLambda = lambdaTerm;
    if (gpuLambda) {
      setAlchemy(ff);
    }
    if ("ASPC".equalsIgnoreCase(ff.getString("SCF_PREDICTOR", "NONE"))) {
      check(call(() -> (int) FfxCuda.SET_SCF_PREDICTOR.invokeExact(handle, 1)));
    }
    // The parent computes the bonded terms only.
    super.setEnergyTermState(STATE.FAST);
    logger.info(" vdW and AMOEBA PME on the GPU (libffxcuda.so)");
  }

  // ---------------------------------------------------------------------------------------
  // OpenMMEnergy's overrides (OpenMMEnergy.java:275-623).

  @Override
  public double energy(double[] x) {
    return energy(x, false);
  }

  @Override
  public double energy(double[] x, boolean verbose) {
    double e = (termState == STATE.SLOW) ? 0.0 : super.energy(x, verbose);   // bonded, CPU
    if (termState == STATE.FAST) {
      return e;
    }
    unscaleCoordinates(x);
    copyIn(x);
    check(call(() -> (int) FfxCuda.SET_COORDINATES.invokeExact(handle, xyz)));
    check(call(() -> (int) FfxCuda.ENERGY.invokeExact(handle, 0, terms, MemorySegment.NULL, counts)));
    scaleCoordinates(x);
    return e + gpuTotal(verbose);
  }

  @Override
  public double energyAndGradient(double[] x, double[] g) {
    return energyAndGradient(x, g, false);
  }

  @Override
  public double energyAndGradient(double[] x, double[] g, boolean verbose) {
    double e = 0.0;
    if (termState == STATE.SLOW) {
      java.util.Arrays.fill(g, 0.0);
    } else {
      e = super.energyAndGradient(x, g, verbose);   // bonded terms; x and g come back scaled
    }
    if (termState == STATE.FAST) {
      return e;
    }
    unscaleCoordinates(x);
    copyIn(x);
    check(call(() -> (int) FfxCuda.ENERGY_AND_GRADIENT.invokeExact(handle, xyz, terms, grad, counts)));
    scaleCoordinates(x);
    double[] scaling = getScaling();
    for (int i = 0; i < 3 * nAtoms; i++) {
      double gi = grad.getAtIndex(JAVA_DOUBLE, i);
      g[i] += (scaling == null) ? gi : gi / scaling[i];
    }
    return e + gpuTotal(verbose);
  }

  /** The gradient at the current coordinates (re-evaluated, as OpenMMEnergy.getGradient does). */
  @Override
  public double[] getGradient(double[] g) {
    if (g == null || g.length < 3 * nAtoms) {
      g = new double[3 * nAtoms];
    }
    double[] x = getCoordinates(null);
    scaleCoordinates(x);
    energyAndGradient(x, g, false);
    unscaleCoordinates(x);
    return g;
  }

  @Override
  public Platform getPlatform() {
    return Platform.FFX;   // a new Platform value (FFX_CUDA) selects this class in energyFactory
  }

  @Override
  public void setCoordinates(double[] x) {
    super.setCoordinates(x);
    copyIn(x);
    check(call(() -> (int) FfxCuda.SET_COORDINATES.invokeExact(handle, xyz)));
  }

  @Override
  public void setCrystal(Crystal crystal) {
    super.setCrystal(crystal);
    Crystal unit = crystal.getUnitCell();
    box3.setAtIndex(JAVA_DOUBLE, 0, unit.a);
    box3.setAtIndex(JAVA_DOUBLE, 1, unit.b);
    box3.setAtIndex(JAVA_DOUBLE, 2, unit.c);
    angles3.setAtIndex(JAVA_DOUBLE, 0, unit.alpha);
    angles3.setAtIndex(JAVA_DOUBLE, 1, unit.beta);
    angles3.setAtIndex(JAVA_DOUBLE, 2, unit.gamma);
    check(call(() -> (int) FfxCuda.SET_BOX.invokeExact(handle, box3, angles3, MemorySegment.NULL)));
  }

  @Override
  public void setLambda(double lambda) {
    super.setLambda(lambda);
    if (gpuLambda) {
      check(call(() -> (int) FfxCuda.SET_LAMBDA.invokeExact(handle, lambda)));
    }
  }

  @Override
  public double getdEdL() {
    double d = super.getdEdL();
    if (gpuLambda && termState != STATE.FAST) {
      check(call(() -> (int) FfxCuda.GET_DEDL.invokeExact(handle, dEdL, d2EdL2, MemorySegment.NULL)));
      d += dEdL.get(JAVA_DOUBLE, 0);
    }
    return d;
  }

  @Override
  public double getd2EdL2() {
    double d = super.getd2EdL2();
    if (gpuLambda && termState != STATE.FAST) {
      check(call(() -> (int) FfxCuda.GET_DEDL.invokeExact(handle, dEdL, d2EdL2, MemorySegment.NULL)));
      d += d2EdL2.get(JAVA_DOUBLE, 0);
    }
    return d;
  }

  @Override
  public void getdEdXdL(double[] gradients) {
    super.getdEdXdL(gradients);
    if (gpuLambda && termState != STATE.FAST) {
      check(call(() -> (int) FfxCuda.GET_DEDL.invokeExact(handle, dEdL, d2EdL2, lambdaGrad)));
      for (int i = 0; i < 3 * nAtoms; i++) {
        gradients[i] += lambdaGrad.getAtIndex(JAVA_DOUBLE, i);
      }
    }
  }

  /** New parameter values of the same atoms (OpenMMEnergy.updateParameters, :623-631). */
  public void updateParameters(Atom[] changed) {
    fillSystem(systemStruct);
    check(call(() -> (int) FfxCuda.UPDATE_PARAMETERS.invokeExact(handle, systemStruct)));
  }

  /** RESPA splits: FAST = bonded on the CPU, SLOW = vdW + PME on the GPU, BOTH = all. */
  @Override
  public void setEnergyTermState(STATE state) {
    termState = state;
    super.setEnergyTermState(STATE.FAST);
  }

  @Override
  public STATE getEnergyTermState() {
    return termState;
  }

  /** Induced dipoles of the last evaluation: ParticleMeshEwald.inducedDipole[0] and inducedDipoleCR[0]. */
  public void getInducedDipoles(double[][] u, double[][] uCR) {
    MemorySegment a = arena.allocate(JAVA_DOUBLE, 3L * nAtoms), b = arena.allocate(JAVA_DOUBLE, 3L * nAtoms);
    check(call(() -> (int) FfxCuda.GET_INDUCED.invokeExact(handle, a, b)));
    for (int i = 0; i < nAtoms; i++) {
      for (int d = 0; d < 3; d++) {
        u[i][d] = a.getAtIndex(JAVA_DOUBLE, 3L * i + d);
        uCR[i][d] = b.getAtIndex(JAVA_DOUBLE, 3L * i + d);
      }
    }
  }

  @Override
  public boolean destroy() {
    boolean ok = super.destroy();
    if (!handle.equals(MemorySegment.NULL)) {
      MemorySegment h = handle;
      call(() -> {
        FfxCuda.DESTROY.invokeExact(h);
        return 0;
      });
      handle = MemorySegment.NULL;
    }
    arena.close();
    return ok;
  }

  // ---------------------------------------------------------------------------------------

  private double gpuTotal(boolean verbose) {
    double e = terms.getAtIndex(JAVA_DOUBLE, FfxCuda.TERM_TOTAL);
    if (verbose) {
      logger.info(String.format(" GPU vdW %16.8f  permanent %16.8f  polarization %16.8f",
          terms.getAtIndex(JAVA_DOUBLE, FfxCuda.TERM_VDW), terms.getAtIndex(JAVA_DOUBLE, FfxCuda.TERM_PERMANENT),
          terms.getAtIndex(JAVA_DOUBLE, FfxCuda.TERM_POLARIZATION)));
    }
    return e;
  }

  private void copyIn(double[] x) {
    if (x.length != 3 * nAtoms) {
      throw new EnergyException(" libffxcuda evaluates every atom: inactive atoms are not supported");
    }
    MemorySegment.copy(x, 0, xyz, JAVA_DOUBLE, 0, x.length);
  }

  /** Status to EnergyException, as PCGSolver.java:554-568 and RealSpaceEnergyRegion.java:384-391 throw. */
  private void check(int st) {
    if (st == FfxCuda.OK) {
      return;
    }
    String msg = FfxCuda.lastError(handle);
    if (st == FfxCuda.ERR_RANGE) {
      logger.warning(" " + msg);   // results complete; only bitwise reproducibility is lost
      return;
    }
    throw new EnergyException(" libffxcuda: " + msg + " (status " + st + ")", false);
  }

  private interface Native {
    int run() throws Throwable;
  }

  private static int call(Native f) {
    try {
      return f.run();
    } catch (Throwable t) {
      throw new EnergyException(" libffxcuda call failed: " + t);
    }
  }

  // ---------------------------------------------------------------------------------------
  // Resolution of the system into the C ABI's arrays, from the objects ParticleMeshEwald and
  // VanDerWaals resolved (ParticleMeshEwald.getMultipoleType / getPolarizeType / getAxisAtoms
  // / getPolarization11, :963-1179; VanDerWaalsForm.getCombinedInverseRmin / getCombinedEps,
  // VanDerWaalsForm.java:534-567; Atom.get12List .. get15List, Atom.java:763-843).

  private static VarHandle field(String name) {
    return FfxCuda.SYSTEM.varHandle(PathElement.groupElement(name));
  }

  private MemorySegment doubles(double[] a) {
    MemorySegment s = arena.allocate(JAVA_DOUBLE, Math.max(1, a.length));
    MemorySegment.copy(a, 0, s, JAVA_DOUBLE, 0, a.length);
    return s;
  }

  private MemorySegment ints(int[] a) {
    MemorySegment s = arena.allocate(JAVA_INT, Math.max(1, a.length));
    MemorySegment.copy(a, 0, s, JAVA_INT, 0, a.length);
    return s;
  }

  /** CSR (ptr[n+1], idx) of per-atom index lists. */
  private int[][] csr(List<int[]> rows) {
    int[] ptr = new int[rows.size() + 1];
    for (int i = 0; i < rows.size(); i++) {
      ptr[i + 1] = ptr[i] + rows.get(i).length;
    }
    int[] idx = new int[ptr[rows.size()]];
    for (int i = 0; i < rows.size(); i++) {
      System.arraycopy(rows.get(i), 0, idx, ptr[i], rows.get(i).length);
    }
    return new int[][] {ptr, idx};
  }

  private static int[] indices(List<Atom> list) {
    int[] r = new int[list.size()];
    for (int k = 0; k < r.length; k++) {
      r[k] = list.get(k).getXyzIndex() - 1;
    }
    return r;
  }

  private void fillSystem(MemorySegment s) {
    ParticleMeshEwald pme = getPmeNode();
    VanDerWaals vdw = getVdwNode();
    VanDerWaalsForm form = vdw.getVDWForm();
    int n = nAtoms;
    double[] x = new double[3 * n], mp = new double[10 * n], pol = new double[n], thole = new double[n];
    double[] pdamp = new double[n], redFactor = new double[n];
    int[] frame = new int[n], axis = new int[3 * n], vtype = new int[n], redParent = new int[n];
    int[][] axisAtoms = pme.getAxisAtoms();
    int[][] ip11 = pme.getPolarization11();
    Map<Integer, Integer> classIndex = new HashMap<>();
    List<Integer> classes = new ArrayList<>();
    List<int[]> m12 = new ArrayList<>(), m13 = new ArrayList<>(), m14 = new ArrayList<>(), m15 = new ArrayList<>();
    List<int[]> g11 = new ArrayList<>();
    for (int i = 0; i < n; i++) {
      Atom a = atoms[i];
      x[3 * i] = a.getX();
      x[3 * i + 1] = a.getY();
      x[3 * i + 2] = a.getZ();
      MultipoleType mt = pme.getMultipoleType(i);
      double[] m = mt.getMultipole();                // e, e*A, e*A^2 (converted from Bohr)
      System.arraycopy(m, 0, mp, 10 * i, 10);
      frame[i] = mt.frameDefinition.ordinal();       // NONE, ZONLY, ZTHENX, BISECTOR, ZTHENBISECTOR, THREEFOLD
      for (int k = 0; k < 3; k++) {
        axis[3 * i + k] = (axisAtoms[i] != null && k < axisAtoms[i].length) ? axisAtoms[i][k] : -1;
      }
      PolarizeType pt = pme.getPolarizeType(i);
      pol[i] = (pt != null) ? pt.polarizability : 0.0;
      thole[i] = (pt != null) ? pt.thole : 0.0;
      pdamp[i] = (pt != null && pt.thole != 0.0) ? Math.pow(pt.polarizability, 1.0 / 6.0) : 0.0;
      int cls = a.getVDWType().atomClass;
      Integer t = classIndex.get(cls);
      if (t == null) {
        t = classes.size();
        classIndex.put(cls, t);
        classes.add(cls);
      }
      vtype[i] = t;
      double rf = a.getVDWType().reductionFactor;
      redParent[i] = i;
      redFactor[i] = 0.0;
      if (rf > 0.0 && a.getNumBonds() == 1) {       // hydrogen reduction toward its heavy atom
        redParent[i] = a.get12List().get(0).getXyzIndex() - 1;
        redFactor[i] = rf;
      }
      m12.add(indices(a.get12List()));
      m13.add(indices(a.get13List()));
      m14.add(indices(a.get14List()));
      m15.add(indices(a.get15List()));
      g11.add(ip11 != null && ip11[i] != null ? ip11[i] : new int[] {i});
    }
    int nt = classes.size();
    double[] inv = new double[nt * nt], eps = new double[nt * nt];
    for (int p = 0; p < nt; p++) {
      for (int q = 0; q < nt; q++) {
        inv[p * nt + q] = form.getCombinedInverseRmin(classes.get(p), classes.get(q));
        eps[p * nt + q] = form.getCombinedEps(classes.get(p), classes.get(q));
      }
    }
    field("n_atoms").set(s, 0L, n);
    field("xyz").set(s, 0L, doubles(x));
    field("multipole").set(s, 0L, doubles(mp));
    field("frame").set(s, 0L, ints(frame));
    field("axis").set(s, 0L, ints(axis));
    field("polarizability").set(s, 0L, doubles(pol));
    field("thole").set(s, 0L, doubles(thole));
    field("pdamp").set(s, 0L, doubles(pdamp));
    field("vdw_type").set(s, 0L, ints(vtype));
    field("red_parent").set(s, 0L, ints(redParent));
    field("red_factor").set(s, 0L, doubles(redFactor));
    field("n_vdw_types").set(s, 0L, nt);
    field("vdw_inv_rmin").set(s, 0L, doubles(inv));
    field("vdw_eps").set(s, 0L, doubles(eps));
    String[] names = {"mask12", "mask13", "mask14", "mask15", "ip11"};
    List<List<int[]>> lists = List.of(m12, m13, m14, m15, g11);
    for (int k = 0; k < names.length; k++) {
      int[][] c = csr(lists.get(k));
      field(names[k] + "_ptr").set(s, 0L, ints(c[0]));
      field(names[k] + "_idx").set(s, 0L, ints(c[1]));
    }
  }

  private static VarHandle param(String name) {
    return FfxCuda.PARAMS.varHandle(PathElement.groupElement(name));
  }

  private void fillParams(MemorySegment p, ForceField ff, Crystal crystal) {
    Crystal unit = crystal.getUnitCell();
    MemorySegment boxSeg = p.asSlice(0, 24);
    boxSeg.setAtIndex(JAVA_DOUBLE, 0, unit.a);
    boxSeg.setAtIndex(JAVA_DOUBLE, 1, unit.b);
    boxSeg.setAtIndex(JAVA_DOUBLE, 2, unit.c);
    MemorySegment angSeg = p.asSlice(232, 24);
    angSeg.setAtIndex(JAVA_DOUBLE, 0, unit.alpha);
    angSeg.setAtIndex(JAVA_DOUBLE, 1, unit.beta);
    angSeg.setAtIndex(JAVA_DOUBLE, 2, unit.gamma);
    ParticleMeshEwald pme = getPmeNode();
    param("vdw_cutoff").set(p, 0L, ff.getDouble("VDW_CUTOFF", 12.0));
    param("vdw_taper").set(p, 0L, ff.getDouble("VDW_TAPER", 0.9));
    param("ewald_cutoff").set(p, 0L, pme.getEwaldCutoff());
    param("ewald_alpha").set(p, 0L, ff.getDouble("EWALD_ALPHA", 0.545));
    param("list_buffer").set(p, 0L, ff.getDouble("LIST_BUFFER", 2.0));
    String[] grid = ff.getString("PME_GRID", "-1 -1 -1").trim().split(" +");
    int gx = Integer.parseInt(grid[0]);
    int gy = grid.length > 1 ? Integer.parseInt(grid[1]) : gx, gz = grid.length > 2 ? Integer.parseInt(grid[2]) : gx;
    MemorySegment g = p.asSlice(64, 12);
    g.setAtIndex(JAVA_INT, 0, gx);
    g.setAtIndex(JAVA_INT, 1, gy);
    g.setAtIndex(JAVA_INT, 2, gz);
    param("pme_order").set(p, 0L, ff.getInteger("PME_ORDER", 5));
    param("polar_eps").set(p, 0L, pme.getPolarEps());
    param("max_scf_iter").set(p, 0L, ff.getInteger("MAX_SCF_ITER", 1000));
    int polar = switch (pme.getPolarizationType()) {
      case NONE -> FfxCuda.POLAR_NONE;
      case DIRECT -> FfxCuda.POLAR_DIRECT;
      default -> FfxCuda.POLAR_MUTUAL;
    };
    param("polarization").set(p, 0L, polar);
    param("precond_cutoff").set(p, 0L, ff.getDouble("CG_PRECONDITIONER_CUTOFF", 4.5));
    param("precond_scale").set(p, 0L, ff.getDouble("CG_PRECONDITIONER_SCALE", 2.0));
    param("electric").set(p, 0L, ff.getDouble("ELECTRIC", 332.0637133));
    param("m12").set(p, 0L, ff.getDouble("MPOLE_12_SCALE", 0.0));
    param("m13").set(p, 0L, ff.getDouble("MPOLE_13_SCALE", 0.0));
    param("m14").set(p, 0L, ff.getDouble("MPOLE_14_SCALE", 0.4));
    param("m15").set(p, 0L, ff.getDouble("MPOLE_15_SCALE", 0.8));
    param("p12").set(p, 0L, ff.getDouble("POLAR_12_SCALE", 0.0));
    param("p13").set(p, 0L, ff.getDouble("POLAR_13_SCALE", 0.0));
    param("p14").set(p, 0L, ff.getDouble("POLAR_14_SCALE", 1.0));
    param("p15").set(p, 0L, ff.getDouble("POLAR_15_SCALE", 1.0));
    param("intra14").set(p, 0L, ff.getDouble("POLAR_14_INTRA", 0.5));
    param("d11").set(p, 0L, ff.getDouble("DIRECT_11_SCALE", 0.0));
    param("v12").set(p, 0L, ff.getDouble("VDW_12_SCALE", 0.0));
    param("v13").set(p, 0L, ff.getDouble("VDW_13_SCALE", 0.0));
    param("v14").set(p, 0L, ff.getDouble("VDW_14_SCALE", 1.0));
    param("precision").set(p, 0L,
        "MIXED".equalsIgnoreCase(ff.getString("CUDA_PRECISION", "FP64")) ? FfxCuda.PRECISION_MIXED
            : FfxCuda.PRECISION_FP64);
  }

  /** Soft atoms (Atom.applyLambda) and the lambda keys read by VanDerWaals and AlchemicalParameters. */
  private void setAlchemy(ForceField ff) {
    int[] soft = new int[nAtoms], mol = new int[nAtoms];
    for (int i = 0; i < nAtoms; i++) {
      soft[i] = atoms[i].applyLambda() ? 1 : 0;
      mol[i] = atoms[i].getMoleculeNumber();
    }
    MemorySegment a = arena.allocate(FfxCuda.ALCHEMY);
    FfxCuda.ALCHEMY.varHandle(PathElement.groupElement("soft")).set(a, 0L, ints(soft));
    FfxCuda.ALCHEMY.varHandle(PathElement.groupElement("molecule")).set(a, 0L, ints(mol));
    setD(a, "vdw_lambda_alpha", ff.getDouble("VDW_LAMBDA_ALPHA", 0.25));
    setD(a, "vdw_lambda_exponent", ff.getDouble("VDW_LAMBDA_EXPONENT", 3.0));
    setD(a, "vdw_lambda_end", ff.getDouble("VDW_LAMBDA_END", 1.0));
    setI(a, "intermolecular_softcore", ff.getBoolean("INTERMOLECULAR_SOFTCORE", false) ? 1 : 0);
    setI(a, "intramolecular_softcore", ff.getBoolean("INTRAMOLECULAR_SOFTCORE", false) ? 1 : 0);
    setI(a, "elec", ff.getBoolean("ELEC_LAMBDATERM", false) ? 1 : 0);
    setD(a, "permanent_lambda_alpha", ff.getDouble("PERMANENT_LAMBDA_ALPHA", 2.0));
    setD(a, "permanent_lambda_exponent", ff.getDouble("PERMANENT_LAMBDA_EXPONENT", 3.0));
    setD(a, "permanent_lambda_start", ff.getDouble("PERMANENT_LAMBDA_START", 0.4));
    setD(a, "permanent_lambda_end", ff.getDouble("PERMANENT_LAMBDA_END", 1.0));
    setD(a, "polarization_lambda_start", ff.getDouble("POLARIZATION_LAMBDA_START", 0.75));
    setD(a, "polarization_lambda_end", ff.getDouble("POLARIZATION_LAMBDA_END", 1.0));
    setD(a, "polarization_lambda_exponent", ff.getDouble("POLARIZATION_LAMBDA_EXPONENT", 3.0));
    setI(a, "ligand_vapor_elec", ff.getBoolean("LIGAND_VAPOR_ELEC", true) ? 1 : 0);
    setI(a, "no_ligand_condensed_scf", ff.getBoolean("NO_LIGAND_CONDENSED_SCF", true) ? 1 : 0);
    check(call(() -> (int) FfxCuda.SET_ALCHEMY.invokeExact(handle, a)));
  }

  private static void setD(MemorySegment a, String name, double v) {
    FfxCuda.ALCHEMY.varHandle(PathElement.groupElement(name)).set(a, 0L, v);
  }

  private static void setI(MemorySegment a, String name, int v) {
    FfxCuda.ALCHEMY.varHandle(PathElement.groupElement(name)).set(a, 0L, v);
  }
}
