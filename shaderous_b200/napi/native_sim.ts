// The hydro part of the reference's Simulation interface (src/sim.ts:465-628) on the B200 library,
// through the N-API addon beside this file (shaderous_addon.cc). A maintainer copies this file to
// src/native_sim.ts and builds the addon with node-gyp; createSim (src/create.ts:58-61) then
// returns a NativeSim (uniform grid) or NativeAmrSim (cfg.amrLevels > 0) for runs whose physics the
// library covers: ideal gas, no gravity, MHD, species, radiation, cooling or sources.
//
// The WebGPU-facing members (device, paramBuffer, clockBuffer, encoders, display resources) have
// no counterpart on this path: the state lives in the library's CUDA buffers. encodeSteps() is
// replaced by step(): callers that batch steps through encoders (api.ts run) call run() instead,
// which the library implements with the same options and result. Members for features outside
// the hydro step throw, naming the feature.
import { createRequire } from 'node:module';
import type { SimConfig, Diagnostics } from './sim';
import type { RunOptions, RunResult } from './ui/api';

const native = createRequire(import.meta.url)('../shaderous_b200/napi/build/Release/shaderous_b200.node');

/** The covered configuration, in the addon's terms (shaderous_addon.cc ToConfig). */
function nativeConfig(cfg: SimConfig): Record<string, unknown> {
  if (cfg.eos !== 'ideal') throw new Error(`NativeSim: the equation of state ${cfg.eos} is not on the native path`);
  if (cfg.gravity !== 'off') throw new Error('NativeSim: gravity is not on the native path');
  return {
    n: cfg.n, ndim: cfg.ndim, box: cfg.problem.box, eosParams: { gamma: cfg.eosParams.gamma },
    bcLo: cfg.bcLo, bcHi: cfg.bcHi, cfl: cfg.cfl, rhoFloor: cfg.rhoFloor, pFloor: cfg.pFloor,
    etaDual: cfg.etaDual, shockThresh: cfg.shockThresh, limiter: cfg.limiter, riemann: cfg.riemann,
    isentropicRecon: cfg.isentropicRecon, tEnd: cfg.tEnd,
  };
}

function unsupported(what: string): never {
  throw new Error(`NativeSim: ${what} is not on the native hydro path`);
}

/** Members common to the uniform and the block grid. */
abstract class NativeBase {
  cfg: SimConfig;
  cur = 0;
  speciesCur = 0;
  readonly speciesStride = 0;
  readonly preparing = false;
  readonly massCount = 0;
  protected h: any;

  constructor(cfg: SimConfig) {
    this.cfg = cfg;
  }
  get n(): number { return this.cfg.n; }
  get nz(): number { return this.cfg.ndim === 3 ? this.cfg.n : 1; }

  /** Take up to `count` steps (encodeSteps' job, without an encoder); returns how many. */
  step(count: number): number {
    this.h.step(count);
    return count;
  }
  /** run() (src/ui/api.ts:538): steps / until / timeoutMs, the same RunResult. */
  run(opts: RunOptions): RunResult { return this.h.run(opts) as RunResult; }
  submitted(): void {}
  stepsResume(): Promise<void> | null { return null; }
  async readDiagnostics(): Promise<Diagnostics | null> { return this.diagnostics(); }
  async diagnostics(): Promise<Diagnostics> { return this.h.diagnostics() as Diagnostics; }
  async runToEnd(batch = 256, maxSteps = Infinity): Promise<number> {
    const r = this.h.run(Number.isFinite(maxSteps) ? { steps: maxSteps, until: this.cfg.tEnd } : { until: this.cfg.tEnd });
    void batch;  // the library paces its own batches (about 50 ms of GPU time each)
    return r.steps;
  }
  writeParams(): void {}
  async buildHydro(): Promise<void> {}
  refreshPotential(): void {}
  status(): string { return `B200 native (${native.version})`; }
  destroy(): void { this.h.destroy(); }

  encodeBrush(): void { unsupported('brush editing'); }
  async placeStar(): Promise<void> { unsupported('placing stars'); }
  async settleStar(): Promise<string> { unsupported('settling stars'); }
  massChanged(): void {}
  addMass(): boolean { return false; }
  async readMasses() { return null; }
  removeAddedMasses(): void {}
  setTracerFixed(): void { unsupported('point masses'); }
  removeMasses(): void { unsupported('point masses'); }
  async readGasLumps() { return null; }
  retuneMasses(): void {}
  async probe() { return null; }
  setSources(list: unknown[]): void { if (list.length) unsupported('sources and sinks'); }
  async debris() { return null; }
  async debrisLedger() { return null; }
}

/** A uniform grid (Sim, src/sim.ts:1938). */
export class NativeSim extends NativeBase {
  constructor(cfg: SimConfig) {
    super(cfg);
    this.h = new native.Sim(nativeConfig(cfg));
  }
  /** Load a built-in problem's initial conditions: { kind, a, axis, seed } (SHZ_PROB_*). */
  reset(problem?: { kind: string; a: number[]; axis?: number; seed?: number }): void {
    if (problem) this.h.resetProblem(problem);
  }
  /** The state as readState() gives it (src/sim.ts:3790-3808): two Float32Arrays of 4 floats a cell. */
  readState(): { u1: Float32Array; u2: Float32Array } { return this.h.readState(); }
  setState(u1: Float32Array, u2: Float32Array): void { this.h.setState(u1, u2); }
}

/** A block grid (AmrSim, src/amr/amr_sim.ts:178). */
export class NativeAmrSim extends NativeBase {
  autoRegrid = true;
  autoBins = true;
  onRegrid?: (steps: number[][]) => void;

  constructor(cfg: SimConfig & { nr?: number; refineHi?: number; refineLo?: number }) {
    super(cfg);
    this.h = new native.AmrSim({ ...nativeConfig(cfg), amrLevels: cfg.amrLevels, amrBudget: cfg.amrBudget,
      timeBins: cfg.timeBins, timeBinsAlways: cfg.timeBinsAlways, nr: cfg.nr, refineHi: cfg.refineHi,
      refineLo: cfg.refineLo });
  }
  reset(problem?: { kind: string; a: number[]; axis?: number; seed?: number }): void {
    if (problem) this.h.resetProblem(problem);
  }
  /** The leaf blocks as corner and side in fractions of the box, and a version (blockBoxes). */
  blockBoxes(): { version: number; boxes: Float32Array } {
    const l = this.h.leaves();
    const nr = (this.cfg as any).nr ?? 2;
    const boxes = new Float32Array(4 * l.count);
    for (let i = 0; i < l.count; i++) {
      const side = 1 / (nr * (1 << l.levels[i]));
      boxes[4 * i] = l.coords[3 * i] * side;
      boxes[4 * i + 1] = l.coords[3 * i + 1] * side;
      boxes[4 * i + 2] = l.coords[3 * i + 2] * side;
      boxes[4 * i + 3] = side;
    }
    return { version: l.count, boxes };
  }
  /** Re-mesh now from the Löhner indicators (AmrSim's refinement check). */
  regrid(): boolean { return this.h.regrid(); }
  readLeaves(): { u1: Float32Array; u2: Float32Array } { return this.h.readLeaves(); }
  table(): Int32Array { return this.h.table(); }
}
