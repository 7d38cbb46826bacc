// FFM binding of libffxcuda.so (include/ffxcuda.h) for Force Field X.
//
// Not compiled in this repository: no JDK is installed on the build machine.  It targets the
// JDK 22+ Foreign Function & Memory API (java.lang.foreign), which the reference's JDK 25
// requirement (pom.xml) provides.  Every downcall handle below names one symbol of the
// header with its C signature; the struct layouts follow the header's field order with the
// padding of the x86-64 / aarch64 C ABI (tests/test_cabi.py pins the same offsets for the
// Python mirror).
package ffx.potential.cuda;

import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_DOUBLE;
import static java.lang.foreign.ValueLayout.JAVA_INT;
import static java.lang.foreign.ValueLayout.JAVA_LONG;

import java.lang.foreign.Arena;
import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.Linker;
import java.lang.foreign.MemoryLayout;
import java.lang.foreign.MemorySegment;
import java.lang.foreign.StructLayout;
import java.lang.foreign.SymbolLookup;
import java.lang.invoke.MethodHandle;

/** Downcall handles and struct layouts of the C ABI. */
public final class FfxCuda {

  private FfxCuda() {}

  /** Status codes (ffxg_status). */
  public static final int OK = 0, ERR_BAD_ARG = 1, ERR_CUDA = 2, ERR_SCF_DIVERGED = 3, ERR_SCF_MAXITER = 4,
      ERR_NONFINITE = 5, ERR_CAPACITY = 6, ERR_RANGE = 7;

  /** Energy terms (FFXG_TERM_*) and counts (FFXG_COUNT_*). */
  public static final int TERM_VDW = 0, TERM_PERMANENT = 1, TERM_POLARIZATION = 2, TERM_TOTAL = 9, N_TERMS = 10;
  public static final int COUNT_VDW = 0, COUNT_PERMANENT = 1, COUNT_SCF_ITER = 2, N_COUNTS = 6;

  /** ffxg_precision and ffxg_polarization. */
  public static final int PRECISION_FP64 = 0, PRECISION_MIXED = 1;
  public static final int POLAR_NONE = 0, POLAR_DIRECT = 1, POLAR_MUTUAL = 2;

  static final Linker LINKER = Linker.nativeLinker();
  static final SymbolLookup LIB =
      SymbolLookup.libraryLookup(System.getProperty("ffx.cuda.library", "libffxcuda.so"), Arena.global());

  private static MethodHandle fn(String name, FunctionDescriptor d) {
    return LINKER.downcallHandle(LIB.find(name).orElseThrow(() -> new UnsatisfiedLinkError(name)), d);
  }

  /** ffxg_system, 192 bytes. */
  public static final StructLayout SYSTEM = MemoryLayout.structLayout(
      JAVA_INT.withName("n_atoms"), MemoryLayout.paddingLayout(4),
      ADDRESS.withName("xyz"), ADDRESS.withName("multipole"), ADDRESS.withName("frame"),
      ADDRESS.withName("axis"), ADDRESS.withName("polarizability"), ADDRESS.withName("thole"),
      ADDRESS.withName("pdamp"), ADDRESS.withName("vdw_type"), ADDRESS.withName("red_parent"),
      ADDRESS.withName("red_factor"),
      JAVA_INT.withName("n_vdw_types"), MemoryLayout.paddingLayout(4),
      ADDRESS.withName("vdw_inv_rmin"), ADDRESS.withName("vdw_eps"),
      ADDRESS.withName("mask12_ptr"), ADDRESS.withName("mask12_idx"),
      ADDRESS.withName("mask13_ptr"), ADDRESS.withName("mask13_idx"),
      ADDRESS.withName("mask14_ptr"), ADDRESS.withName("mask14_idx"),
      ADDRESS.withName("mask15_ptr"), ADDRESS.withName("mask15_idx"),
      ADDRESS.withName("ip11_ptr"), ADDRESS.withName("ip11_idx"));

  /** ffxg_params, 256 bytes. */
  public static final StructLayout PARAMS = MemoryLayout.structLayout(
      MemoryLayout.sequenceLayout(3, JAVA_DOUBLE).withName("box"),
      JAVA_DOUBLE.withName("vdw_cutoff"), JAVA_DOUBLE.withName("vdw_taper"),
      JAVA_DOUBLE.withName("ewald_cutoff"), JAVA_DOUBLE.withName("ewald_alpha"),
      JAVA_DOUBLE.withName("list_buffer"),
      MemoryLayout.sequenceLayout(3, JAVA_INT).withName("pme_grid"), JAVA_INT.withName("pme_order"),
      JAVA_DOUBLE.withName("polar_eps"), JAVA_INT.withName("max_scf_iter"), JAVA_INT.withName("polarization"),
      JAVA_DOUBLE.withName("precond_cutoff"), JAVA_DOUBLE.withName("precond_scale"),
      JAVA_DOUBLE.withName("electric"),
      JAVA_DOUBLE.withName("m12"), JAVA_DOUBLE.withName("m13"), JAVA_DOUBLE.withName("m14"),
      JAVA_DOUBLE.withName("m15"),
      JAVA_DOUBLE.withName("p12"), JAVA_DOUBLE.withName("p13"), JAVA_DOUBLE.withName("p14"),
      JAVA_DOUBLE.withName("p15"),
      JAVA_DOUBLE.withName("intra14"), JAVA_DOUBLE.withName("d11"),
      JAVA_DOUBLE.withName("v12"), JAVA_DOUBLE.withName("v13"), JAVA_DOUBLE.withName("v14"),
      JAVA_INT.withName("precision"), MemoryLayout.paddingLayout(4),
      MemoryLayout.sequenceLayout(3, JAVA_DOUBLE).withName("angles"));

  /** ffxg_alchemy, 112 bytes. */
  public static final StructLayout ALCHEMY = MemoryLayout.structLayout(
      ADDRESS.withName("soft"), ADDRESS.withName("molecule"),
      JAVA_DOUBLE.withName("vdw_lambda_alpha"), JAVA_DOUBLE.withName("vdw_lambda_exponent"),
      JAVA_DOUBLE.withName("vdw_lambda_end"),
      JAVA_INT.withName("intermolecular_softcore"), JAVA_INT.withName("intramolecular_softcore"),
      JAVA_INT.withName("elec"), MemoryLayout.paddingLayout(4),
      JAVA_DOUBLE.withName("permanent_lambda_alpha"), JAVA_DOUBLE.withName("permanent_lambda_exponent"),
      JAVA_DOUBLE.withName("permanent_lambda_start"), JAVA_DOUBLE.withName("permanent_lambda_end"),
      JAVA_DOUBLE.withName("polarization_lambda_start"), JAVA_DOUBLE.withName("polarization_lambda_end"),
      JAVA_DOUBLE.withName("polarization_lambda_exponent"),
      JAVA_INT.withName("ligand_vapor_elec"), JAVA_INT.withName("no_ligand_condensed_scf"));

  // int ffxg_create(const ffxg_system*, const ffxg_params*, ffxg_handle**)
  public static final MethodHandle CREATE = fn("ffxg_create",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS));
  // void ffxg_destroy(ffxg_handle*)
  public static final MethodHandle DESTROY = fn("ffxg_destroy", FunctionDescriptor.ofVoid(ADDRESS));
  // const char* ffxg_last_error(const ffxg_handle*)
  public static final MethodHandle LAST_ERROR = fn("ffxg_last_error", FunctionDescriptor.of(ADDRESS, ADDRESS));
  // int ffxg_set_coordinates(ffxg_handle*, const double* xyz)
  public static final MethodHandle SET_COORDINATES = fn("ffxg_set_coordinates",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
  // int ffxg_set_box(ffxg_handle*, const double box[3], const double angles[3], const int32_t pme_grid[3])
  public static final MethodHandle SET_BOX = fn("ffxg_set_box",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS));
  // int ffxg_update_parameters(ffxg_handle*, const ffxg_system*)
  public static final MethodHandle UPDATE_PARAMETERS = fn("ffxg_update_parameters",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
  // int ffxg_energy(ffxg_handle*, int want_grad, double* terms, double* grad, int64_t* counts)
  public static final MethodHandle ENERGY = fn("ffxg_energy",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT, ADDRESS, ADDRESS, ADDRESS));
  // int ffxg_energy_and_gradient(ffxg_handle*, const double* xyz, double* terms, double* grad, int64_t* counts)
  public static final MethodHandle ENERGY_AND_GRADIENT = fn("ffxg_energy_and_gradient",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS, ADDRESS));
  // int ffxg_get_induced_dipoles(ffxg_handle*, double* u, double* u_cr)
  public static final MethodHandle GET_INDUCED = fn("ffxg_get_induced_dipoles",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS));
  // int ffxg_set_alchemy(ffxg_handle*, const ffxg_alchemy*)
  public static final MethodHandle SET_ALCHEMY = fn("ffxg_set_alchemy",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
  // int ffxg_set_lambda(ffxg_handle*, double)
  public static final MethodHandle SET_LAMBDA = fn("ffxg_set_lambda",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_DOUBLE));
  // int ffxg_get_dEdL(ffxg_handle*, double* dEdL, double* d2EdL2, double* dEdXdL)
  public static final MethodHandle GET_DEDL = fn("ffxg_get_dEdL",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS));
  // int ffxg_set_scf_predictor(ffxg_handle*, int)
  public static final MethodHandle SET_SCF_PREDICTOR = fn("ffxg_set_scf_predictor",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, JAVA_INT));
  // int ffxg_param_grad(ffxg_handle*, double* dEdM, double* dEdalpha)
  public static final MethodHandle PARAM_GRAD = fn("ffxg_param_grad",
      FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS));

  /** The C string behind a const char* (UTF-8, NUL-terminated). */
  static String cString(MemorySegment p) {
    if (p.equals(MemorySegment.NULL)) {
      return "";
    }
    return p.reinterpret(Long.MAX_VALUE).getString(0);
  }

  /** ffxg_last_error(h) as a Java string. */
  public static String lastError(MemorySegment handle) {
    try {
      MemorySegment p = (MemorySegment) LAST_ERROR.invokeExact(handle);
      return cString(p);
    } catch (Throwable t) {
      return "ffxg_last_error failed: " + t;
    }
  }

  /** int64_t counts[FFXG_N_COUNTS]. */
  public static final MemoryLayout COUNTS = MemoryLayout.sequenceLayout(N_COUNTS, JAVA_LONG);
}
