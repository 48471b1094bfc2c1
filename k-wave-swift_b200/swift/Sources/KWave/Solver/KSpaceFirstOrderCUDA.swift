// KSpaceFirstOrderCUDA.swift — the `DeviceKind.cuda` path of k-wave-swift: kspaceFirstOrder and its
// adjoint run by libkwave_cuda.so (hand-written sm_100a CUDA) through the C ABI of kwave_cuda.h.
//
// This file joins the KWave target of a k-wave-swift checkout (Sources/KWave/Solver/), next to
// KSpaceFirstOrder.swift, with three edits to that package:
//   Package.swift      .systemLibrary(name: "CKWaveCUDA", path: "Sources/CKWaveCUDA") next to
//                      CHDF5 (Package.swift:17-21), and "CKWaveCUDA" in the KWave target's
//                      dependencies;
//   KWave.swift        DeviceKind (KWave.swift:12-22) gains `case cuda` (its `stream` maps it to
//                      .cpu: MLX only holds the inputs and outputs of a CUDA run);
//   KSpaceFirstOrder   kspaceFirstOrder (KSpaceFirstOrder.swift:79-107) starts with
//                      `if options.device == .cuda { return kspaceFirstOrderCUDA(...) }`.
// Everything the solver reads is flattened into one kw_sim_desc of host buffers (MLXArray ->
// [Float], row-major like MLX), the library copies them to the device, runs every time step and
// returns each requested SimulationOutput field in the reference's shapes. Errors come back as
// kw_status codes with a message; like the reference's preconditions they stop the program.
import CKWaveCUDA
import Foundation
import MLX

// MARK: - host buffers

/// Owns the host copies a descriptor points at until the library has copied them.
private final class HostBuffers {
    private var owned: [UnsafeMutablePointer<Float>] = []

    func floats(_ a: MLXArray) -> [Float] { a.asType(.float32).asArray(Float.self) }

    func copy(_ v: [Float]) -> UnsafePointer<Float> {
        let p = UnsafeMutablePointer<Float>.allocate(capacity: max(v.count, 1))
        p.initialize(from: v, count: v.count)
        owned.append(p)
        return UnsafePointer(p)
    }

    func array(_ a: MLXArray?) -> kw_array {
        guard let a else { return kw_array(data: nil, len: 0) }
        let v = floats(a)
        return kw_array(data: copy(v), len: v.count)
    }

    func grid(_ a: MLXArray?) -> UnsafePointer<Float>? {
        guard let a else { return nil }
        return copy(floats(a))
    }

    /// A source signal: 1-D is one broadcast row, 2-D one row per source point (signalRows,
    /// KSpaceFirstOrder.swift:179-189).
    func signal(_ a: MLXArray?) -> kw_signal {
        guard let a else { return kw_signal(data: nil, rows: 0, len: 0) }
        let rows = a.ndim <= 1 ? 1 : a.shape[0]
        let len = a.ndim <= 1 ? a.size : a.shape[1]
        return kw_signal(data: copy(floats(a)), rows: Int32(rows), len: Int32(len))
    }

    deinit { for p in owned { p.deallocate() } }
}

private func sourceMode(_ m: SourceMode) -> Int32 {
    switch m {
    case .dirichlet: return Int32(KW_SOURCE_DIRICHLET.rawValue)
    case .additive: return Int32(KW_SOURCE_ADDITIVE.rawValue)
    case .additiveNoCorrection: return Int32(KW_SOURCE_ADDITIVE_NO_CORRECTION.rawValue)
    }
}

private func absorptionMode(_ m: AbsorptionMode) -> Int32 {
    switch m {
    case .noAbsorption: return Int32(KW_ABSORPTION_NONE.rawValue)
    case .powerLaw: return Int32(KW_ABSORPTION_POWER_LAW.rawValue)
    case .noDispersion: return Int32(KW_ABSORPTION_NO_DISPERSION.rawValue)
    case .stokes: return Int32(KW_ABSORPTION_STOKES.rawValue)
    }
}

/// The reference's grid, medium, source, sensor and options as one descriptor.
private func makeDescriptor(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource, sensor: KWaveSensor,
                            options: SimulationOptions, buffers: HostBuffers) -> kw_sim_desc {
    var d = kw_sim_desc()
    kw_sim_desc_init(&d)
    d.dim = Int32(grid.dim)
    d.nx = Int32(grid.nx); d.ny = Int32(grid.ny); d.nz = Int32(grid.nz)
    d.dx = grid.dx; d.dy = grid.dy; d.dz = grid.dz
    d.dt = grid.dt; d.nt = Int32(grid.nt)
    switch options.pmlSize { case let .uniform(m): d.pml_size = Int32(m) }
    d.pml_alpha = options.pmlAlpha
    d.smooth_p0 = options.smoothP0 ? 1 : 0
    d.smooth_c0 = options.smoothC0 ? 1 : 0
    d.smooth_rho0 = options.smoothRho0 ? 1 : 0

    d.sound_speed = buffers.array(medium.soundSpeed)
    d.density = buffers.array(medium.density)
    d.alpha_coeff = buffers.array(medium.alphaCoeff)
    d.alpha_power = medium.alphaPower ?? .nan
    d.alpha_mode = absorptionMode(medium.alphaMode)
    d.b_on_a = buffers.array(medium.bOnA)

    d.p0 = buffers.grid(source.p0)
    d.p_mask = buffers.grid(source.pMask)
    d.p = buffers.signal(source.p)
    d.p_mode = sourceMode(source.pMode)
    d.u_mask = buffers.grid(source.uMask)
    d.ux = buffers.signal(source.ux)
    d.uy = buffers.signal(source.uy)
    d.uz = buffers.signal(source.uz)
    d.u_mode = sourceMode(source.uMode)

    d.record = UInt32(sensor.record.rawValue)
    if let mask = sensor.mask {
        // Cartesian when the mask is [dim, nPoints] (Recording.swift:51), else a binary grid mask
        if mask.ndim == 2 && mask.dim(0) == grid.dim {
            d.sensor_kind = Int32(KW_SENSOR_CARTESIAN.rawValue)
            d.sensor_points = Int32(mask.dim(1))
        } else {
            d.sensor_kind = Int32(KW_SENSOR_BINARY.rawValue)
        }
        d.sensor_mask = buffers.grid(mask)
    }
    d.directivity_angle = buffers.grid(sensor.directivityAngle)
    d.directivity_size = sensor.directivitySize ?? .nan
    d.directivity_pattern = sensor.directivityPattern == .pressure
        ? Int32(KW_DIRECTIVITY_PRESSURE.rawValue) : Int32(KW_DIRECTIVITY_GRADIENT.rawValue)
    return d
}

// MARK: - context and errors

/// One library context (a CUDA device and its stream) per call, like the reference's per-call
/// MLX stream use.
private final class CUDAContext {
    let handle: OpaquePointer

    init(device: Int32 = 0) {
        var h: OpaquePointer?
        let st = kw_context_create(device, &h)
        guard st == 0, let h else {
            fatalError("kspaceFirstOrderCUDA: kw_context_create failed (\(st)): \(String(cString: kw_last_error_message(nil)))")
        }
        handle = h
    }

    func check(_ status: Int32, _ what: String) {
        precondition(status == 0, "\(what): kw_status \(status): \(String(cString: kw_last_error_message(handle)))")
    }

    deinit { kw_context_destroy(handle) }
}

/// Closures of SimulationOptions reached from the library's C callbacks.
private final class CallbackBox {
    let progress: ((Int, Int) -> Void)?
    let monitor: ((Int, MLXArray) -> Void)?
    let shape: [Int]

    init(options: SimulationOptions, shape: [Int]) {
        progress = options.progress
        monitor = options.fieldMonitor
        self.shape = shape
    }
}

private func gridShape(_ grid: KWaveGrid) -> [Int] {
    switch grid.dim {
    case 1: return [grid.nx]
    case 2: return [grid.nx, grid.ny]
    default: return [grid.nx, grid.ny, grid.nz]
    }
}

// MARK: - kspaceFirstOrder on the GPU

/// kspaceFirstOrder (KSpaceFirstOrder.swift:79-107) run by libkwave_cuda.so. Same arguments and
/// result; `options.device == .cuda` routes here.
public func kspaceFirstOrderCUDA(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                                 sensor: KWaveSensor, options: SimulationOptions = .init()) -> SimulationOutput {
    precondition(grid.nt > 0, "call grid.makeTime(...) before running the solver")
    let ctx = CUDAContext()
    let buffers = HostBuffers()
    var d = makeDescriptor(grid: grid, medium: medium, source: source, sensor: sensor, options: options,
                           buffers: buffers)
    var sim: OpaquePointer?
    ctx.check(kw_sim_create(ctx.handle, &d, &sim), "kw_sim_create")
    guard let sim else { fatalError("kw_sim_create returned no simulation") }
    defer { kw_sim_destroy(sim) }

    let shape = gridShape(grid)
    let box = CallbackBox(options: options, shape: shape)
    var cb = kw_callbacks()
    if options.progress != nil {
        cb.progress = { t, nt, user in
            let b = Unmanaged<CallbackBox>.fromOpaque(user!).takeUnretainedValue()
            b.progress?(Int(t), Int(nt))
        }
    }
    if options.fieldMonitor != nil {
        cb.monitor = { t, p, count, user in
            let b = Unmanaged<CallbackBox>.fromOpaque(user!).takeUnretainedValue()
            b.monitor?(Int(t), MLXArray(Array(UnsafeBufferPointer(start: p, count: count)), b.shape))
        }
    }
    cb.monitor_interval = Int32(max(options.fieldMonitorInterval, 1))
    cb.user = Unmanaged.passUnretained(box).toOpaque()
    ctx.check(withExtendedLifetime(box) { kw_sim_run(sim, &cb) }, "kw_sim_run")

    var nSensor: Int32 = 0
    ctx.check(kw_sim_num_sensor_points(sim, &nSensor), "kw_sim_num_sensor_points")
    var steps: Int32 = 0
    ctx.check(kw_sim_current_step(sim, &steps), "kw_sim_current_step")

    // one output field in the reference's shape: series [nSensor, nt], aggregates [nSensor],
    // final fields the grid's shape (Recording.swift:129-168)
    func field(_ f: kw_field, _ kind: Int) -> MLXArray? {
        var n = 0
        ctx.check(kw_sim_output_size(sim, Int32(f.rawValue), &n), "kw_sim_output_size")
        if n == 0 { return nil }
        var host = [Float](repeating: 0, count: n)
        ctx.check(host.withUnsafeMutableBufferPointer { kw_sim_get_output(sim, Int32(f.rawValue), $0.baseAddress, n) },
                  "kw_sim_get_output")
        switch kind {
        case 0: return MLXArray(host, [Int(nSensor), Int(steps)])
        case 1: return MLXArray(host, [Int(nSensor)])
        default: return MLXArray(host, shape)
        }
    }
    var out = SimulationOutput()
    out.p = field(KW_FIELD_P, 0)
    out.pMax = field(KW_FIELD_P_MAX, 1)
    out.pMin = field(KW_FIELD_P_MIN, 1)
    out.pRms = field(KW_FIELD_P_RMS, 1)
    out.pFinal = field(KW_FIELD_P_FINAL, 2)
    out.ux = field(KW_FIELD_UX, 0)
    out.uy = field(KW_FIELD_UY, 0)
    out.uz = field(KW_FIELD_UZ, 0)
    out.uxMax = field(KW_FIELD_UX_MAX, 1)
    out.uyMax = field(KW_FIELD_UY_MAX, 1)
    out.uzMax = field(KW_FIELD_UZ_MAX, 1)
    out.uxRms = field(KW_FIELD_UX_RMS, 1)
    out.uyRms = field(KW_FIELD_UY_RMS, 1)
    out.uzRms = field(KW_FIELD_UZ_RMS, 1)
    out.uxFinal = field(KW_FIELD_UX_FINAL, 2)
    out.uyFinal = field(KW_FIELD_UY_FINAL, 2)
    out.uzFinal = field(KW_FIELD_UZ_FINAL, 2)
    out.ixAvg = field(KW_FIELD_IX_AVG, 1)
    out.iyAvg = field(KW_FIELD_IY_AVG, 1)
    out.izAvg = field(KW_FIELD_IZ_AVG, 1)
    return out
}

/// kspaceFirstOrderAS (KSpaceFirstOrderAS.swift:19-309) run by libkwave_cuda.so: the same
/// descriptor with its axisymmetric flag set (2D, x axial, y radial).
public func kspaceFirstOrderASCUDA(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                                   sensor: KWaveSensor, options: SimulationOptions = .init()) -> SimulationOutput {
    precondition(grid.dim == 2, "axisymmetric solver requires a 2D grid (x axial, y radial)")
    let ctx = CUDAContext()
    let buffers = HostBuffers()
    var d = makeDescriptor(grid: grid, medium: medium, source: source, sensor: sensor, options: options,
                           buffers: buffers)
    d.axisymmetric = 1
    var sim: OpaquePointer?
    ctx.check(kw_sim_create(ctx.handle, &d, &sim), "kw_sim_create")
    guard let sim else { fatalError("kw_sim_create returned no simulation") }
    defer { kw_sim_destroy(sim) }
    ctx.check(kw_sim_run(sim, nil), "kw_sim_run")
    var nSensor: Int32 = 0, steps: Int32 = 0
    ctx.check(kw_sim_num_sensor_points(sim, &nSensor), "kw_sim_num_sensor_points")
    ctx.check(kw_sim_current_step(sim, &steps), "kw_sim_current_step")
    var out = SimulationOutput()
    for (f, isSeries) in [(KW_FIELD_P, true), (KW_FIELD_P_FINAL, false)] {
        var n = 0
        ctx.check(kw_sim_output_size(sim, Int32(f.rawValue), &n), "kw_sim_output_size")
        if n == 0 { continue }
        var host = [Float](repeating: 0, count: n)
        ctx.check(host.withUnsafeMutableBufferPointer { kw_sim_get_output(sim, Int32(f.rawValue), $0.baseAddress, n) },
                  "kw_sim_get_output")
        if isSeries { out.p = MLXArray(host, [Int(nSensor), Int(steps)]) }
        else { out.pFinal = MLXArray(host, [grid.nx, grid.ny]) }
    }
    return out
}

// MARK: - adjoint

/// Checkpoint schedule of the adjoint's reverse sweep (kw_checkpoint_policy).
public enum CheckpointPolicy {
    case sqrtNt
    case interval(Int)
    case memoryBudget(bytes: Double)
    case storeAll
}

/// Gradients of the sensor-data misfit L = 1/2 sum (p_sensor - data)^2 of kspaceFirstOrder with
/// respect to the sound speed, the density (`gradRho0`) and (with `source.p0`) the initial
/// pressure, by the discrete adjoint of the time step (no counterpart in the reference). `data`
/// has the p output's shape [nSensor, nt].
public func kspaceFirstOrderAdjoint(grid: KWaveGrid, medium: KWaveMedium, source: KWaveSource,
                                    sensor: KWaveSensor, data: MLXArray, options: SimulationOptions = .init(),
                                    gradP0: Bool = false, gradRho0: Bool = false, policy: CheckpointPolicy = .sqrtNt)
    -> (misfit: Double, gradC0: MLXArray, gradP0: MLXArray?, gradRho0: MLXArray?) {
    let ctx = CUDAContext()
    let buffers = HostBuffers()
    var d = makeDescriptor(grid: grid, medium: medium, source: source, sensor: sensor, options: options,
                           buffers: buffers)
    var a = kw_adjoint_desc()
    kw_adjoint_desc_init(&a)
    switch policy {
    case .sqrtNt: a.policy = Int32(KW_CHECKPOINT_SQRT.rawValue)
    case let .interval(k): a.policy = Int32(KW_CHECKPOINT_INTERVAL.rawValue); a.checkpoint_interval = Int32(k)
    case let .memoryBudget(bytes): a.policy = Int32(KW_CHECKPOINT_BUDGET.rawValue); a.memory_budget = bytes
    case .storeAll: a.policy = Int32(KW_CHECKPOINT_STORE_ALL.rawValue)
    }
    let n = grid.totalGridPoints
    let observed = buffers.floats(data)
    var gc = [Float](repeating: 0, count: n)
    var gp = [Float](repeating: 0, count: gradP0 ? n : 0)
    var gr = [Float](repeating: 0, count: gradRho0 ? n : 0)
    let status: Int32 = observed.withUnsafeBufferPointer { op in
        gc.withUnsafeMutableBufferPointer { gcp in
            gp.withUnsafeMutableBufferPointer { gpp in
                gr.withUnsafeMutableBufferPointer { grp in
                    a.data = op.baseAddress
                    a.grad_c0 = gcp.baseAddress
                    a.grad_p0 = gradP0 ? gpp.baseAddress : nil
                    a.grad_rho0 = gradRho0 ? grp.baseAddress : nil
                    return kw_adjoint_run(ctx.handle, &d, &a)
                }
            }
        }
    }
    ctx.check(status, "kw_adjoint_run")
    let shape = gridShape(grid)
    return (a.misfit, MLXArray(gc, shape), gradP0 ? MLXArray(gp, shape) : nil, gradRho0 ? MLXArray(gr, shape) : nil)
}
