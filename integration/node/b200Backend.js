// The `b200` compute backend: the reference's backend contract
// (js_fdtd/src/backends/CONTRACT.md:104-137, types.js:27-33) over the N-API
// module of binding_b200.cpp, which wraps libfdtd_b200.so.
//
// Install as js_fdtd/src/backends/b200/b200Backend.js with the addon built to
// js_fdtd/src/backends/b200/build/Release/fdtd_b200.node (binding.gyp beside
// this file) and register it in registry.js (registry.patch).
//
// run(problem) advances the whole time loop on the GPU.  It uploads the
// problem the reference already built (scenario.js:73-131: grid, coeffs,
// cpml, sources, samplers, ff), runs `options.batchSize` steps per call, copies
// the port traces into samplers.*.sampled_value after each batch and yields a
// progress snapshot (cudaBackend.js:254-290 does the same per batch), and at
// the end fills ff.<array>.re / .im in place, as accumulateFarfieldDFT would
// have (CONTRACT.md:130-132).  Precision: problem.options.precision 'f64'
// (default, the bit-faithful drop-in of the wasm-cpu path) or 'f32'.
import { createRequire } from 'module';

const require = createRequire(import.meta.url);
let addon = null;
try {
  addon = require('./build/Release/fdtd_b200.node');
} catch {
  addon = null;
}

// Coefficient ids of fdtd_ctx_upload_coeff (the reference's COEFF_ORDER,
// cudaBackend.js:53-60).
const COEFF_ORDER = ['Cexe', 'Cexhz', 'Cexhy', 'Ceye', 'Ceyhx', 'Ceyhz', 'Ceze', 'Cezhy', 'Cezhx',
                     'Chxh', 'Chxey', 'Chxez', 'Chyh', 'Chyez', 'Chyex', 'Chzh', 'Chzex', 'Chzey'];
// Far-field accumulator ids of fdtd_ctx_read_farfield.
const FF_ORDER = ['cjyxp', 'cjzxp', 'cjyxn', 'cjzxn', 'cjxyp', 'cjzyp', 'cjxyn', 'cjzyn',
                  'cjxzp', 'cjyzp', 'cjxzn', 'cjyzn', 'cmyxp', 'cmzxp', 'cmyxn', 'cmzxn',
                  'cmxyp', 'cmzyp', 'cmxyn', 'cmzyn', 'cmxzp', 'cmyzp', 'cmxzn', 'cmyzn'];
const FACES = ['xn', 'xp', 'yn', 'yp', 'zn', 'zp'];
const DIR = { x: 0, y: 1, z: 2 };
const PRECISION = { f64: 0, f32: 1 };

// captureSampledCurrents (sampling.js:204-245) as one ordered gather list
// (component, flat index, weight): the same terms in the same order, with the
// signs folded into the weights.  The device sums the list from zero in order,
// so the current is bit-identical to the reference's.
export function currentList(obs, g) {
  const comp = [], idx = [], w = [];
  const s = obs.direction[1] === 'n' ? -1 : 1;
  const hx = (i, j, k) => (i * g.ny + j) * g.nz + k;
  const hy = (i, j, k) => (i * g.nyp1 + j) * g.nz + k;
  const hz = (i, j, k) => (i * g.ny + j) * g.nzp1 + k;
  const I = obs.is - 1, J = obs.js - 1, K = obs.ks - 1;
  const IE = obs.ie - 1, JE = obs.je - 1, KE = obs.ke - 1;
  const add = (c, n, d) => { comp.push(c); idx.push(n); w.push(s * d); };
  switch (obs.direction[0]) {
    case 'x': {
      const ix = IE - 1;
      for (let j = J; j <= JE - 1; j++) add(1, hy(ix, j, K - 1), g.dy);
      for (let k = K; k <= KE - 1; k++) add(2, hz(ix, JE - 1, k), g.dz);
      for (let j = J; j <= JE - 1; j++) add(1, hy(ix, j, KE - 1), -g.dy);
      for (let k = K; k <= KE - 1; k++) add(2, hz(ix, J - 1, k), -g.dz);
      break;
    }
    case 'y': {
      const jx = JE - 1;
      for (let k = K; k <= KE - 1; k++) add(2, hz(I - 1, jx, k), g.dz);
      for (let i = I; i <= IE - 1; i++) add(0, hx(i, jx, KE - 1), g.dx);
      for (let k = K; k <= KE - 1; k++) add(2, hz(IE, jx, k), -g.dz);
      for (let i = I; i <= IE - 1; i++) add(0, hx(i, jx, K - 1), -g.dx);
      break;
    }
    default: {
      const kx = KE - 1;
      for (let i = I; i <= IE - 1; i++) add(0, hx(i, J - 1, kx), g.dx);
      for (let j = J; j <= JE - 1; j++) add(1, hy(IE, j, kx), g.dy);
      for (let i = I; i <= IE - 1; i++) add(0, hx(i, JE, kx), -g.dx);
      for (let j = J; j <= JE - 1; j++) add(1, hy(I - 1, j, kx), -g.dy);
    }
  }
  return [Int32Array.from(comp), Int32Array.from(idx), Float64Array.from(w)];
}

function upload(h, problem) {
  const { grid, coeffs, cpml, samplers, sources, ff } = problem;
  COEFF_ORDER.forEach((name, w) => addon.uploadCoeff(h, w, Float64Array.from(coeffs[name])));
  FACES.forEach((f, id) => { if (cpml[f]) addon.uploadCpml(h, id, cpml[f]); });
  for (const vs of sources.voltageSources ?? []) {
    const axis = vs.direction[0];
    const coef = axis === 'x' ? vs.Cexs : axis === 'y' ? vs.Ceys : vs.Cezs;
    addon.addVSource(h, DIR[axis], Int32Array.from(vs.field_indices), Float64Array.from(coef),
                     Float64Array.from(vs.voltage_per_e_field));
  }
  for (const sv of samplers.sampledVoltages ?? [])
    addon.addSVoltage(h, DIR[sv.direction[0]], Int32Array.from(sv.field_indices), sv.Csvf);
  for (const si of samplers.sampledCurrents ?? []) addon.addSCurrent(h, ...currentList(si, grid));
  if (ff && ff.nFreq > 0) addon.setupFarfield(h, ff);
}

export default {
  name: 'b200',

  async isAvailable() {
    try {
      return !!addon && addon.deviceCount() > 0;
    } catch {
      return false;
    }
  },

  meta() {
    return { name: 'b200', precision: ['f64', 'f32'], farfield: 'device' };
  },

  async *run(problem) {
    const { grid, samplers, ff, options = {} } = problem;
    const batchSize = options.batchSize ?? 50;
    const total = grid.numberOfTimeSteps;
    const precision = PRECISION[options.precision ?? 'f64'];
    if (precision === undefined) throw new Error(`b200: unknown precision "${options.precision}"`);
    const h = addon.create({ ...grid, precision, device: options.device ?? 0 });
    try {
      upload(h, problem);
      const sv = samplers.sampledVoltages ?? [], si = samplers.sampledCurrents ?? [];
      const t0 = Date.now();
      for (let ts = 0; ts < total;) {
        const n = Math.min(batchSize, total - ts);
        addon.run(h, n);
        ts += n;
        sv.forEach((o, q) => addon.readTrace(h, 0, q, o.sampled_value.subarray(0, ts)));
        si.forEach((o, q) => addon.readTrace(h, 1, q, o.sampled_value.subarray(0, ts)));
        const elapsed = (Date.now() - t0) / 1000;
        yield {
          step: ts, total, elapsed, percent: (ts / total * 100).toFixed(1),
          voltage: sv.length > 0 ? sv[0].sampled_value[ts - 1] : null,
          time_ns: (ts - 0.5) * grid.dt * 1e9, backend: 'b200',
        };
        await new Promise(r => setTimeout(r, 0));
      }
      const st = addon.status(h);
      if (st.code !== 0) throw new Error(`b200: non-finite field at step ${st.step}`);
      if (ff && ff.nFreq > 0) FF_ORDER.forEach((name, a) => addon.readFarfield(h, a, ff[name].re, ff[name].im));
    } finally {
      addon.free(h);
    }
  },
};
