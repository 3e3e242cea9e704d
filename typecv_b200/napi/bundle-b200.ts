// bundleAdjustGpu over libtba.so: the B200 drop-in for TypeCV's WebGPU operator
// (src/sfm/bundle/gpu/bundle.ts:803-839, joint-focal.ts:78-929), to be placed beside it as
// src/sfm/bundle/gpu/bundle-b200.ts.  UNBUILT HERE: this image and its GPU hosts have no Node or
// TypeScript toolchain; the same C ABI is exercised from Python by the tests of this repository.
//
// What stays the reference's: option and problem validation (bundleProblem), packing
// (packBundleScene, finiteGpuArray), and reading the output (checkBundleOutput, bundleOutputPose,
// bundleOutputLandmarks, bundleOutputReport, separateBundleDirections), imported unchanged.  What
// changes: the device plan between packing and reading is one addon call (tba_napi.c ->
// tba_bundle_adjust), run on a libuv worker thread; the output array has the layout the reference
// reads (poses, points, 26 state words, and the log focal scale on the shared-focal route).
import { createRequire } from 'node:module';
import type { SparseReconstruction } from '../../../contracts/scene.ts';
import { finiteGpuArray } from '../../../geometry/gpu/bounds.ts';
import { separateBundleDirections } from '../bundle-directions.ts';
import { bundleStallTolerance } from '../bundle-shared.ts';
import {
  bundleArraySizes,
  bundleOutputLandmarks,
  bundleOutputPose,
  bundleOutputReport,
  bundleProblem,
  checkBundleOutput,
  packBundleScene,
  snapshotBundleModel,
} from './bundle-host.ts';
import {
  BUNDLE_STATE,
  type GpuBundleAdjustmentOptions,
  type GpuBundleAdjustmentResult,
} from './bundle-shared.ts';

interface TbaControl {
  cameras: number;
  points: number;
  directionalPoints: number;
  observations: number;
  anchor: number;
  scaleView: number;
  iterations: number;
  maxCg: number;
  sharedFocal: boolean;
  precision: 'fp64' | 'mixed';
  huber: number;
  cgTolerance: number;
  stallTolerance: number;
}

interface TbaAddon {
  openDevice(ordinal: number): unknown;
  closeDevice(device: unknown): void;
  bundleAdjustPacked(
    device: unknown,
    control: TbaControl,
    scene: Float64Array,
    index: Uint32Array,
  ): Promise<Float64Array>;
}

const addon = createRequire(import.meta.url)('typecv-b200/build/Release/tba_napi.node') as TbaAddon;

/** A CUDA device handle of libtba.so (one stream; calls on it run one at a time). */
export interface B200Device {
  readonly native: unknown;
  close(): void;
}

export function openB200Device(ordinal = 0): B200Device {
  const native = addon.openDevice(ordinal);
  return { native, close: () => addon.closeDevice(native) };
}

export interface B200BundleOptions extends GpuBundleAdjustmentOptions {
  /** 'mixed': FP32 Jacobian factors and Schur product inside the FP64 LM loop (no reference counterpart). */
  readonly precision?: 'fp64' | 'mixed';
}

/** The reference operator's option checks (bundle.ts:808-838); the options that select WebGPU
 *  plans are accepted and have no effect on the B200 engine. */
function checkOptions(input: SparseReconstruction, options: B200BundleOptions): void {
  const size = options.cameraProductWorkgroupSize;
  if (size !== undefined && ![32, 64, 128, 256, 'auto'].includes(size))
    throw new RangeError('cameraProductWorkgroupSize must be 32, 64, 128, 256 or auto');
  const tile = options.cameraProductTileSize;
  if (tile !== undefined && (!Number.isSafeInteger(tile) || tile < 1 || tile > 0xffffffff))
    throw new RangeError('cameraProductTileSize must be a positive u32 integer');
  if (options.cameraProduct !== undefined && options.cameraProduct !== 'workgroups' && options.cameraProduct !== 'rows')
    throw new RangeError("cameraProduct must be 'workgroups' or 'rows'");
  if (options.schurCache !== undefined && typeof options.schurCache !== 'boolean')
    throw new RangeError('schurCache must be a boolean');
  const reduction = options.schurReduction;
  if (reduction !== undefined && reduction !== 'auto' && reduction !== 'serial' && reduction !== 'cooperative')
    throw new RangeError('Invalid Schur reduction mode');
  if (options.refineSharedFocal && options.focalGroups) {
    const groups = new Set(input.views.map((v) => options.focalGroups!.get(v.id)));
    if (groups.size > 1) throw new RangeError('Per-group focal refinement is not implemented on the GPU');
  }
  if (options.precision !== undefined && options.precision !== 'fp64' && options.precision !== 'mixed')
    throw new RangeError("precision must be 'fp64' or 'mixed'");
}

/** Jointly optimize camera poses and points (and one shared log-focal scale with
 *  `refineSharedFocal`) on a B200, with the result object of the WebGPU operator. */
export async function bundleAdjustGpu(
  device: B200Device,
  input: SparseReconstruction,
  options: B200BundleOptions = {},
): Promise<GpuBundleAdjustmentResult> {
  checkOptions(input, options);
  const shared = options.refineSharedFocal === true;
  // The two routes' default PCG budgets (bundle.ts:94, joint-focal.ts:83).
  const problem = bundleProblem(input, options, (cameras) =>
    shared ? Math.min(256, Math.max(32, cameras * 12 + 1)) : Math.min(96, Math.max(24, cameras * 12)),
  );
  const { finitePoints, C, P, M, iterations, huber, maxCg, tolerance, byId, anchorId, scaleId, active } = problem;
  const { sceneSize, trialSize, indexSize } = bundleArraySizes(C, P, M);
  const model = snapshotBundleModel(problem.input);
  const { source, indices } = packBundleScene(model, byId, active, { C, P, M, sceneSize, indexSize });
  if (!finiteGpuArray(source)) throw new RangeError('GPU BA input exceeds supported coordinate bounds');
  const started = performance.now();
  const values = await addon.bundleAdjustPacked(
    device.native,
    {
      cameras: C,
      points: P,
      directionalPoints: P - finitePoints,
      observations: M,
      anchor: byId.get(anchorId)!,
      scaleView: byId.get(scaleId)!,
      iterations,
      maxCg,
      sharedFocal: shared,
      precision: options.precision ?? 'fp64',
      huber,
      cgTolerance: tolerance,
      stallTolerance: bundleStallTolerance(options),
    },
    source,
    indices,
  );
  const base = trialSize;
  checkBundleOutput(values, base);
  // Fixed cameras and runs without an accepted step return the inputs' own values.
  const changed = values[base + BUNDLE_STATE.accepted]! > 0;
  const scale = shared && changed ? Math.exp(values[base + BUNDLE_STATE.focalScale]!) : 1;
  const reconstruction: SparseReconstruction = {
    views: model.views.map((view, c) => ({
      ...view,
      camera: scale !== 1 ? { ...view.camera, fx: view.camera.fx * scale, fy: view.camera.fy * scale } : view.camera,
      pose: bundleOutputPose(values, view, c, changed, active),
    })),
    landmarks: bundleOutputLandmarks(model, values, C, changed),
  };
  const elapsed = performance.now() - started;
  return separateBundleDirections(
    {
      reconstruction,
      ...bundleOutputReport(values, base, M),
      // The WebGPU plan report has no counterpart; the call's wall time stands in for its timings.
      execution: { backend: 'cuda', wallMs: elapsed } as unknown as GpuBundleAdjustmentResult['execution'],
    },
    finitePoints,
  );
}
