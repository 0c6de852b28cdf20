package nanoj.liveSRRF;

// Drop-in for the reference's device-engine class nanoj.liveSRRF.LiveSRRF_CL
// (src/nanoj/liveSRRF/LiveSRRF_CL.java:29-1017): the same public constructor, fields and methods,
// with the OpenCL body replaced by downcalls into libesrrf.so (include/esrrf.h) through the
// Foreign Function & Memory API (java.lang.foreign, Java 22+; Java 21 with --enable-preview).
//
// Source only: this file is not compiled in the repository (the build image has no JDK).  The
// drivers (gui/LiveSRRF_optimised_.java, gui/ParametersSweep_.java) keep every call; their only
// change is the import of the device type, com.jogamp.opencl.CLDevice -> the nested
// LiveSRRF_CL.CLDevice below (same getName()).  libesrrf.so is found through the system property
// "esrrf.lib" (a path) or else java.library.path.
//
// Errors: a failed esrrf_create throws RuntimeException as initialise does when OpenCL cannot start
// (LiveSRRF_CL.java:115-119); other failures are logged and execution carries on, as the reference
// does; NaN is zeroed by the library at read-back.

import ij.IJ;
import ij.ImageStack;
import ij.process.FloatProcessor;
import ij.process.ImageProcessor;
import nanoj.core.java.io.LoadNanoJTable;

import java.io.IOException;
import java.lang.foreign.Arena;
import java.lang.foreign.FunctionDescriptor;
import java.lang.foreign.Linker;
import java.lang.foreign.MemoryLayout;
import java.lang.foreign.MemorySegment;
import java.lang.foreign.StructLayout;
import java.lang.foreign.SymbolLookup;
import java.lang.invoke.MethodHandle;
import java.nio.file.Path;
import java.util.Map;

import static java.lang.foreign.MemoryLayout.PathElement.groupElement;
import static java.lang.foreign.ValueLayout.ADDRESS;
import static java.lang.foreign.ValueLayout.JAVA_FLOAT;
import static java.lang.foreign.ValueLayout.JAVA_INT;
import static java.lang.foreign.ValueLayout.JAVA_LONG;
import static java.lang.foreign.ValueLayout.JAVA_SHORT;

public class LiveSRRF_CL {

    // ------------------------------------------------------------------ native bindings

    private static final Linker LINKER = Linker.nativeLinker();
    private static final SymbolLookup LIB = loadLibrary();

    private static SymbolLookup loadLibrary() {
        String path = System.getProperty("esrrf.lib");
        if (path != null) return SymbolLookup.libraryLookup(Path.of(path), Arena.global());
        System.loadLibrary("esrrf");
        return SymbolLookup.loaderLookup();
    }

    private static MethodHandle fn(String name, FunctionDescriptor d) {
        return LINKER.downcallHandle(LIB.find(name).orElseThrow(
                () -> new UnsatisfiedLinkError("libesrrf.so does not export " + name)), d);
    }

    // esrrf_params, in the field order of include/esrrf.h (120 bytes on LP64)
    private static final StructLayout PARAMS = MemoryLayout.structLayout(
            JAVA_INT.withName("width"), JAVA_INT.withName("height"), JAVA_INT.withName("magnification"),
            JAVA_FLOAT.withName("fwhm"), JAVA_INT.withName("sensitivity"),
            JAVA_INT.withName("n_frames_on_gpu"), JAVA_INT.withName("n_frame_for_srrf"),
            JAVA_INT.withName("block_length"), JAVA_INT.withName("device"),
            JAVA_INT.withName("int_weighting"), JAVA_INT.withName("mp_correction"),
            JAVA_INT.withName("interp"), JAVA_INT.withName("fht_scale"), JAVA_INT.withName("kernel"),
            JAVA_INT.withName("frames_per_launch"), JAVA_INT.withName("n_planes"),
            ADDRESS.withName("roi"), ADDRESS.withName("theta_deg"), ADDRESS.withName("shift_x"),
            ADDRESS.withName("shift_y"), ADDRESS.withName("intensity_coeff"),
            JAVA_FLOAT.withName("background"), JAVA_FLOAT.withName("axial_offset_nm"),
            JAVA_FLOAT.withName("pixel_size_um"), MemoryLayout.paddingLayout(4));

    private static final MethodHandle DEVICE_COUNT = fn("esrrf_device_count",
            FunctionDescriptor.of(JAVA_INT, ADDRESS));
    private static final MethodHandle DEVICE_INFO = fn("esrrf_device_info",
            FunctionDescriptor.of(JAVA_INT, JAVA_INT, ADDRESS, JAVA_LONG, ADDRESS, ADDRESS));
    private static final MethodHandle DEFAULTS = fn("esrrf_default_params", FunctionDescriptor.ofVoid(ADDRESS));
    private static final MethodHandle CREATE = fn("esrrf_create", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    private static final MethodHandle DESTROY = fn("esrrf_destroy", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    private static final MethodHandle SET_DRIFT = fn("esrrf_set_drift",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, JAVA_INT));
    private static final MethodHandle RESET = fn("esrrf_reset_frame_position", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    private static final MethodHandle CALC_F32 = fn("esrrf_calculate_srrf_f32",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT));
    private static final MethodHandle CALC_U16 = fn("esrrf_calculate_srrf_u16",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_INT));
    private static final MethodHandle READ = fn("esrrf_read_srrf", FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS));
    private static final MethodHandle SHAPE = fn("esrrf_output_shape",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, ADDRESS, ADDRESS));
    private static final MethodHandle READ_GRAD = fn("esrrf_read_gradients",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG));
    private static final MethodHandle READ_ALIGNED = fn("esrrf_read_aligned_pixels",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG));
    private static final MethodHandle READ_MP = fn("esrrf_read_mp_maps",
            FunctionDescriptor.of(JAVA_INT, ADDRESS, ADDRESS, JAVA_LONG));
    private static final MethodHandle FINISH = fn("esrrf_finish_queue", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    private static final MethodHandle CANCEL = fn("esrrf_request_cancel", FunctionDescriptor.of(JAVA_INT, ADDRESS));
    private static final MethodHandle LAST_ERROR = fn("esrrf_last_error", FunctionDescriptor.of(ADDRESS, ADDRESS));

    private static final int ESRRF_OK = 0, ESRRF_CANCELLED = 1;

    // ------------------------------------------------------------------ device type

    /** A CUDA device as the drivers see an OpenCL one: they list getName() in their dialog and
     *  hand the chosen object back to initialise (gui/LiveSRRF_optimised_.java:157-187). */
    public static final class CLDevice {
        private final int ordinal, computeUnits, clockMHz;
        private final String name;

        CLDevice(int ordinal, String name, int computeUnits, int clockMHz) {
            this.ordinal = ordinal;
            this.name = name;
            this.computeUnits = computeUnits;
            this.clockMHz = clockMHz;
        }

        public String getName() { return name; }
        public int getMaxComputeUnits() { return computeUnits; }
        public int getMaxClockFrequency() { return clockMHz; }
        public int getOrdinal() { return ordinal; }
        @Override public String toString() { return name + " (CUDA " + ordinal + ")"; }
    }

    // ------------------------------------------------------------------ public fields (LiveSRRF_CL.java:41-64, 84)

    public int widthS, heightS,
            nPlanes,
            nPlanesM,
            gradientMag = 2; // the bicubic path's gradient grid factor
    public final int nReconstructions = 3; // AVG, VAR, TAC2
    public ImageStack imsSRRF;
    public CLDevice[] allCLdevices;

    // ------------------------------------------------------------------ state

    private final boolean DEBUG;
    private final Arena arena = Arena.ofShared();
    private MemorySegment handle = MemorySegment.NULL;
    private int widthM, heightM, magnification, nFrameForSRRF;
    private boolean do3DSRRF, doMPmapCorrection, fht;
    private double[] roi3D, intCoeffs3D;
    private float background3D;

    // ------------------------------------------------------------------ members

    /** LiveSRRF_CL(boolean DEBUG) (LiveSRRF_CL.java:105): no device work. */
    public LiveSRRF_CL(boolean DEBUG) {
        this.DEBUG = DEBUG;
    }

    /** checkDevices (LiveSRRF_CL.java:111-155): every CUDA device, fastest (SMs x clock) first. */
    public void checkDevices() {
        try (Arena a = Arena.ofConfined()) {
            MemorySegment n = a.allocate(JAVA_INT);
            if ((int) DEVICE_COUNT.invokeExact(n) != ESRRF_OK) {
                allCLdevices = new CLDevice[0];
                return;
            }
            int count = n.get(JAVA_INT, 0);
            allCLdevices = new CLDevice[count];
            MemorySegment name = a.allocate(256);
            MemorySegment sms = a.allocate(JAVA_INT), clk = a.allocate(JAVA_INT);
            for (int d = 0; d < count; d++) {
                int rc = (int) DEVICE_INFO.invokeExact(d, name, 256L, sms, clk);
                allCLdevices[d] = new CLDevice(d, rc == ESRRF_OK ? name.getString(0) : "CUDA device " + d,
                        sms.get(JAVA_INT, 0), clk.get(JAVA_INT, 0));
                if (DEBUG) IJ.log("Found " + allCLdevices[d] + ": " + sms.get(JAVA_INT, 0) + " SMs, "
                        + clk.get(JAVA_INT, 0) + " MHz");
            }
            java.util.Arrays.sort(allCLdevices, (x, y) -> Long.compare(
                    (long) y.getMaxComputeUnits() * y.getMaxClockFrequency(),
                    (long) x.getMaxComputeUnits() * x.getMaxClockFrequency()));
        } catch (Throwable t) {
            IJ.log("No CUDA device: " + t);
            allCLdevices = new CLDevice[0];
        }
    }

    /** initialise (LiveSRRF_CL.java:159-264): validates, allocates and builds on the device.  A
     *  non-null calibration path means the 3-D (MFM) path, read with NanoJ-Core's table loader as
     *  the reference does (:210-227). */
    public void initialise(int width, int height, int magnification, float fwhm, int sensitivity,
                           int nFramesOnGPU, int nFrameForSRRF, int blockLength, CLDevice chosenDevice,
                           boolean intWeighting, boolean doMPmapCorrection, boolean doFHTinterpolation,
                           String calibTablePath3DSRRF, float axialOffset, float pixelSize) {
        release();
        this.magnification = magnification;
        this.nFrameForSRRF = nFrameForSRRF;
        this.doMPmapCorrection = doMPmapCorrection;
        this.do3DSRRF = calibTablePath3DSRRF != null;
        this.fht = doFHTinterpolation && !do3DSRRF;  // FHT is forced off in 3-D (LiveSRRF_CL.java:166-168)
        try {
            MemorySegment p = arena.allocate(PARAMS);
            DEFAULTS.invokeExact(p);
            setInt(p, "width", width);
            setInt(p, "height", height);
            setInt(p, "magnification", magnification);
            p.set(JAVA_FLOAT, off("fwhm"), fwhm);
            setInt(p, "sensitivity", sensitivity);
            setInt(p, "n_frames_on_gpu", nFramesOnGPU);
            setInt(p, "n_frame_for_srrf", nFrameForSRRF);
            setInt(p, "block_length", blockLength);
            setInt(p, "device", chosenDevice == null ? -1 : chosenDevice.getOrdinal());
            setInt(p, "int_weighting", intWeighting ? 1 : 0);
            setInt(p, "mp_correction", doMPmapCorrection ? 1 : 0);
            setInt(p, "interp", fht ? 0 : 1);
            if (do3DSRRF) {
                Map<String, double[]> t = new LoadNanoJTable(calibTablePath3DSRRF).getData();
                double[] shiftX = t.get("X-shift (pixels)"), shiftY = t.get("Y-shift (pixels)");
                double[] theta = t.get("Theta (degrees)"), axial = t.get("Axial positions");
                roi3D = t.get("ROI #");
                intCoeffs3D = t.get("Intensity scaling");
                background3D = (float) t.get("Background level (ADC)")[0];
                int P = shiftX.length;
                setInt(p, "n_planes", P);
                p.set(ADDRESS, off("roi"), floats(roi3D));
                p.set(ADDRESS, off("theta_deg"), floats(theta));
                p.set(ADDRESS, off("shift_x"), floats(shiftX));
                p.set(ADDRESS, off("shift_y"), floats(shiftY));
                p.set(ADDRESS, off("intensity_coeff"), floats(intCoeffs3D));
                p.set(JAVA_FLOAT, off("background"), background3D);
                double sum = 0;
                for (double z : axial) sum += z;
                if (sum != 0) axialOffset = (float) LinearRegressions.linearRegressionLeastSquareNoOffset(axial);
                IJ.log("3D axial offset: " + axialOffset + " nm");
            }
            p.set(JAVA_FLOAT, off("axial_offset_nm"), axialOffset);
            p.set(JAVA_FLOAT, off("pixel_size_um"), pixelSize);
            MemorySegment out = arena.allocate(ADDRESS);
            int rc = (int) CREATE.invokeExact(p, out);
            if (rc != ESRRF_OK) throw new IllegalStateException(lastError(MemorySegment.NULL));
            handle = out.get(ADDRESS, 0);
            MemorySegment w = arena.allocate(JAVA_INT), h = arena.allocate(JAVA_INT), d = arena.allocate(JAVA_INT);
            check((int) SHAPE.invokeExact(handle, w, h, d), "output shape");
            widthM = w.get(JAVA_INT, 0);
            heightM = h.get(JAVA_INT, 0);
            nPlanesM = d.get(JAVA_INT, 0);
            widthS = widthM / magnification;
            heightS = heightM / magnification;
            nPlanes = do3DSRRF ? nPlanesM / magnification : 1;
            if (DEBUG) IJ.log("widthM/heightM: " + widthM + "/" + heightM + ", planes " + nPlanesM);
        } catch (IOException e) {
            IJ.log("Could not read the calibration table: " + e);
            throw new RuntimeException("Something went wrong initializing the GPU.", e);
        } catch (Throwable t) {
            throw new RuntimeException("Something went wrong initializing the GPU.", t);
        }
    }

    /** prepareBuffersBICinterpolation (LiveSRRF_CL.java:266-459): done by esrrf_create in
     *  initialise; kept for callers that name it. */
    public void prepareBuffersBICinterpolation(int nFramesOnGPU, float fwhm, float sensitivity,
                                               double[] shiftX3D, double[] shiftY3D, double[] theta3D) {
        if (DEBUG) IJ.log("bicubic-path buffers are prepared by initialise");
    }

    /** prepareBuffersFHTinterpolation (LiveSRRF_CL.java:462-579): done by esrrf_create. */
    public void prepareBuffersFHTinterpolation(int nFramesOnGPU, float fwhm, float sensitivity) {
        if (DEBUG) IJ.log("FHT-path buffers are prepared by initialise");
    }

    /** loadDriftXYGPUbuffer (LiveSRRF_CL.java:583-595): per-frame drift of the block in raw pixels
     *  (the library stores it x magnification, as the reference does). */
    public void loadDriftXYGPUbuffer(float[] driftX, float[] driftY) {
        try (Arena a = Arena.ofConfined()) {
            int n = nFrameForSRRF;
            MemorySegment dx = a.allocate(JAVA_FLOAT, n), dy = a.allocate(JAVA_FLOAT, n);
            MemorySegment.copy(driftX, 0, dx, JAVA_FLOAT, 0, Math.min(n, driftX.length));
            MemorySegment.copy(driftY, 0, dy, JAVA_FLOAT, 0, Math.min(n, driftY.length));
            check((int) SET_DRIFT.invokeExact(handle, dx, dy, n), "loadDriftXYGPUbuffer");
        } catch (Throwable t) {
            IJ.log("loadDriftXYGPUbuffer: " + t);
        }
    }

    /** prepareDataFHT_SRRF (LiveSRRF_CL.java:598-633): the Fourier interpolation runs on the GPU
     *  inside calculateSRRF here; nothing to prepare on the host. */
    public void prepareDataFHT_SRRF(ImageStack imsRawData) {
        if (DEBUG) IJ.log("Fourier interpolation runs on the GPU in calculateSRRF");
    }

    /** calculateSRRF (LiveSRRF_CL.java:636-746): accumulates these frames into the current block;
     *  returns true if cancelled (Escape pressed).  16-bit stacks go up as uint16, others as float. */
    public synchronized boolean calculateSRRF(ImageStack imsRawData) {
        if (IJ.escapePressed()) {
            try {
                int ignored = (int) CANCEL.invokeExact(handle);
            } catch (Throwable t) {
            }
            return true;
        }
        int n = imsRawData.getSize(), wh = imsRawData.getWidth() * imsRawData.getHeight();
        boolean u16 = imsRawData.getBitDepth() == 16;
        try (Arena a = Arena.ofConfined()) {
            int rc;
            if (u16) {
                MemorySegment frames = a.allocate(JAVA_SHORT, (long) n * wh);
                for (int f = 0; f < n; f++)
                    MemorySegment.copy((short[]) imsRawData.getPixels(f + 1), 0, frames,
                            JAVA_SHORT, (long) f * wh * 2, wh);
                rc = (int) CALC_U16.invokeExact(handle, frames, n);
            } else {
                MemorySegment frames = a.allocate(JAVA_FLOAT, (long) n * wh);
                for (int f = 0; f < n; f++) {
                    ImageProcessor ip = imsRawData.getProcessor(f + 1);
                    float[] px = (float[]) ip.convertToFloatProcessor().getPixels();
                    MemorySegment.copy(px, 0, frames, JAVA_FLOAT, (long) f * wh * 4, wh);
                }
                rc = (int) CALC_F32.invokeExact(handle, frames, n);
            }
            if (rc == ESRRF_CANCELLED) return true;
            check(rc, "calculateSRRF");
        } catch (Throwable t) {
            IJ.log("calculateSRRF: " + t);
        }
        return false;
    }

    /** readSRRFbuffer (LiveSRRF_CL.java:749-794): finalises VAR/TAC2 (and the MP correction on the
     *  bicubic and 3-D paths) and sets imsSRRF to [AVG, VAR, TAC2, INT] x nPlanesM slices. */
    public void readSRRFbuffer() {
        long plane = (long) widthM * heightM;
        try (Arena a = Arena.ofConfined()) {
            MemorySegment out = a.allocate(JAVA_FLOAT, 4 * nPlanesM * plane);
            check((int) READ.invokeExact(handle, out), "readSRRFbuffer");
            imsSRRF = new ImageStack(widthM, heightM);
            String[] names = {"AVG", "VAR", "TAC2", "INT"};
            for (int k = 0; k < 4; k++)
                for (int z = 0; z < nPlanesM; z++) {
                    float[] px = out.asSlice(((long) k * nPlanesM + z) * plane * 4, plane * 4).toArray(JAVA_FLOAT);
                    imsSRRF.addSlice(names[k] + (nPlanesM > 1 ? " z=" + z : ""), new FloatProcessor(widthM, heightM, px));
                }
        } catch (Throwable t) {
            IJ.log("readSRRFbuffer: " + t);
        }
    }

    /** readGradientBuffers (LiveSRRF_CL.java:797-879): gradient components of the first frame of
     *  the last push. */
    public ImageStack readGradientBuffers() {
        // FHT path: Gx, Gy of the interpolated frame; bicubic and 3-D paths: the components on the
        // 2x gradient grid (x planes in 3-D)
        int comps = do3DSRRF ? 3 : 2;
        int gw = fht ? widthM : gradientMag * widthS, gh = fht ? heightM : gradientMag * heightS;
        return readPlanes(READ_GRAD, comps * nPlanes, gw, gh, "readGradientBuffers");
    }

    /** readAlignedPixels (LiveSRRF_CL.java:881-906): the 3-D path's aligned planes. */
    public ImageStack readAlignedPixels() {
        return readPlanes(READ_ALIGNED, nPlanes, widthS, heightS, "readAlignedPixels");
    }

    /** readMPmaps (LiveSRRF_CL.java:909-935): the macro-pixel maps of the last read. */
    public ImageStack readMPmaps() {
        int M = magnification;
        return readPlanes(READ_MP, 3 * (do3DSRRF ? M : 1), M, M, "readMPmaps");
    }

    /** release (LiveSRRF_CL.java:939-951). */
    public void release() {
        if (handle.equals(MemorySegment.NULL)) return;
        try {
            int ignored = (int) DESTROY.invokeExact(handle);
        } catch (Throwable t) {
            IJ.log("release: " + t);
        }
        handle = MemorySegment.NULL;
    }

    /** resetFramePosition (LiveSRRF_CL.java:955-960): starts a new SR block. */
    public void resetFramePosition() {
        try {
            check((int) RESET.invokeExact(handle), "resetFramePosition");
        } catch (Throwable t) {
            IJ.log("resetFramePosition: " + t);
        }
    }

    /** reshapeImageStack3D (LiveSRRF_CL.java:963-994): the MFM camera frames split into the 3 x 3
     *  plane layout, background subtracted and divided by each plane's intensity scaling.  The
     *  library does the same on the GPU inside calculateSRRF; this host form serves callers that
     *  want the planes themselves. */
    public ImageStack reshapeImageStack3D(ImageStack ims) {
        int W = ims.getWidth(), H = ims.getHeight(), ws = W / 3, hs = H / 3;
        ImageStack out = new ImageStack(ws, hs);
        for (int f = 1; f <= ims.getSize(); f++) {
            ImageProcessor ip = ims.getProcessor(f);
            for (int z = 0; z < nPlanes; z++) {
                int col = ((int) roi3D[z]) % 3, row = ((int) roi3D[z] - col) / 3;
                int x0 = Math.round((float) W / 3 * col), y0 = Math.round((float) H / 3 * row);
                float c = (float) intCoeffs3D[z];
                float[] px = new float[ws * hs];
                for (int y = 0; y < hs; y++)
                    for (int x = 0; x < ws; x++)
                        px[y * ws + x] = (ip.getf(x0 + x, y0 + y) - background3D) / c;
                out.addSlice(new FloatProcessor(ws, hs, px));
            }
        }
        return out;
    }

    /** print3DeSRRFinLog (LiveSRRF_CL.java:996-1006): the 3-D banner. */
    public void print3DeSRRFinLog() {
        IJ.log("---- 3D eSRRF (multi-focus planes) on libesrrf ----");
    }

    /** finishQueue (LiveSRRF_CL.java:1009-1015): waits for every queued kernel and copy. */
    public void finishQueue() {
        if (handle.equals(MemorySegment.NULL)) return;
        try {
            check((int) FINISH.invokeExact(handle), "finishQueue");
        } catch (Throwable t) {
            IJ.log("finishQueue: " + t);
        }
    }

    // ------------------------------------------------------------------ helpers

    private ImageStack readPlanes(MethodHandle h, int planes, int w, int hgt, String what) {
        long n = (long) planes * w * hgt;
        try (Arena a = Arena.ofConfined()) {
            MemorySegment out = a.allocate(JAVA_FLOAT, n);
            check((int) h.invokeExact(handle, out, n), what);
            ImageStack ims = new ImageStack(w, hgt);
            for (int p = 0; p < planes; p++)
                ims.addSlice(new FloatProcessor(w, hgt,
                        out.asSlice((long) p * w * hgt * 4, (long) w * hgt * 4).toArray(JAVA_FLOAT)));
            return ims;
        } catch (Throwable t) {
            IJ.log(what + ": " + t);
            return null;
        }
    }

    private static long off(String field) {
        return PARAMS.byteOffset(groupElement(field));
    }

    private static void setInt(MemorySegment p, String field, int v) {
        p.set(JAVA_INT, off(field), v);
    }

    private MemorySegment floats(double[] v) {
        MemorySegment s = arena.allocate(JAVA_FLOAT, v.length);
        for (int i = 0; i < v.length; i++) s.setAtIndex(JAVA_FLOAT, i, (float) v[i]);
        return s;
    }

    private void check(int rc, String what) {
        if (rc != ESRRF_OK) throw new IllegalStateException(what + ": " + lastError(handle));
    }

    private static String lastError(MemorySegment h) {
        try {
            MemorySegment m = (MemorySegment) LAST_ERROR.invokeExact(h);
            return m.reinterpret(4096).getString(0);
        } catch (Throwable t) {
            return "(no message)";
        }
    }
}
