// N-API module `fdtd_b200` over libfdtd_b200.so (include/fdtd_b200.h).
//
// Shape of the reference's CUDA addon, js_fdtd/src/backends/cuda/native/binding.cpp:
// typed arrays are borrowed as zero-copy views for the duration of a call
// (binding.cpp:51-60), every failing call throws Napi::Error("<call>: " +
// fdtd_last_error()) (binding.cpp:23-26), and the module is registered with
// NODE_API_MODULE (binding.cpp:174-188).  Unlike that addon, which keeps one
// global problem, every problem here is an opaque handle (an External), so
// several problems and batches of them can be live at once.
//
// Exported functions (JS name -> C entry point):
//   deviceCount()                                   fdtd_device_count
//   create({nx,ny,nz,dx,dy,dz,dt,numberOfTimeSteps,precision,device})  fdtd_create
//   free(h)                                         fdtd_free
//   uploadCoeff(h, which, Float64Array)             fdtd_ctx_upload_coeff (COEFF_ORDER ids 0..17)
//   uploadCpml(h, faceId, face)                     fdtd_ctx_upload_cpml (a cpml.js face object)
//   addVSource(h, dir, Int32Array idx, Float64Array coef, Float64Array wave)  fdtd_ctx_add_vsource
//   addSVoltage(h, dir, Int32Array idx, Csvf)       fdtd_ctx_add_svoltage
//   addSCurrent(h, Int32Array comp, Int32Array idx, Float64Array w)  fdtd_ctx_add_scurrent
//   setupFarfield(h, ff)                            fdtd_ctx_setup_farfield (a farfield.js ff object)
//   run(h, count)                                   fdtd_ctx_run
//   step(h)                                         fdtd_ctx_step
//   status(h) -> {code, step}                       fdtd_status
//   readTrace(h, kind, probe, Float64Array out)     fdtd_ctx_read_trace
//   readField(h, which, Float64Array out)           fdtd_ctx_read_field
//   readFarfield(h, array, Float64Array re, Float64Array im)  fdtd_ctx_read_farfield
//   farfieldPost(h, Float64Array theta, Float64Array phi, nFreq) -> {radp, dTheta, dPhi}
//                                                   fdtd_ctx_farfield_post
//   dft(Float64Array x, dt, Float64Array freqs, shift) -> {re, im}  fdtd_dft
//   saveState(h) -> Buffer / loadState(h, Buffer)   fdtd_ctx_state_size / save_state / load_state
//   setDftBlock(h, steps), setDftAccumulator(h, kahan)  fdtd_ctx_set_dft_block / set_dft_accumulator
//   setXWall(h, wall)                               fdtd_ctx_set_x_wall (E at i = nx: 0 reference reads, 1 PEC wall)
//   batchCreate([h...]) -> b, batchRun(b, count), batchShape(b, chunk, rows, prefetch, group,
//   streams, width[, perLaunch]), batchFree(b)      fdtd_batch_*
//
// Built by integration/node/binding.gyp; not compiled in this repository's
// environment, which has no Node.js (tests/test_integration_sources.py checks
// it against the C header with a stand-in napi.h).
#include <napi.h>

#include <string>
#include <vector>

#include "fdtd_b200.h"

namespace {

void Check(Napi::Env env, int rc, const char* what) {
  if (rc != FDTD_OK) throw Napi::Error::New(env, std::string(what) + ": " + fdtd_last_error());
}

fdtd_ctx* Ctx(const Napi::Value& v) { return v.As<Napi::External<fdtd_ctx>>().Data(); }
fdtd_batch* Batch(const Napi::Value& v) { return v.As<Napi::External<fdtd_batch>>().Data(); }

template <class T>
T* Ptr(const Napi::Value& v) {
  return v.As<Napi::TypedArrayOf<T>>().Data();
}
template <class T>
long Len(const Napi::Value& v) {
  return (long)v.As<Napi::TypedArrayOf<T>>().ElementLength();
}
int Int(const Napi::Value& v) { return v.As<Napi::Number>().Int32Value(); }
double Dbl(const Napi::Value& v) { return v.As<Napi::Number>().DoubleValue(); }

Napi::Value DeviceCount(const Napi::CallbackInfo& a) {
  int n = 0;
  if (fdtd_device_count(&n) != FDTD_OK) n = 0;
  return Napi::Number::New(a.Env(), n);
}

Napi::Value Create(const Napi::CallbackInfo& a) {
  Napi::Object o = a[0].As<Napi::Object>();
  FdtdConfig c;
  c.nx = Int(o.Get("nx"));
  c.ny = Int(o.Get("ny"));
  c.nz = Int(o.Get("nz"));
  c.dx = Dbl(o.Get("dx"));
  c.dy = Dbl(o.Get("dy"));
  c.dz = Dbl(o.Get("dz"));
  c.dt = Dbl(o.Get("dt"));
  c.numberOfTimeSteps = Int(o.Get("numberOfTimeSteps"));
  c.precision = o.Has("precision") ? Int(o.Get("precision")) : FDTD_PREC_F64;
  c.device = o.Has("device") ? Int(o.Get("device")) : 0;
  fdtd_ctx* h = nullptr;
  Check(a.Env(), fdtd_create(&c, &h), "create");
  return Napi::External<fdtd_ctx>::New(a.Env(), h);
}

Napi::Value Free(const Napi::CallbackInfo& a) {
  fdtd_free(Ctx(a[0]));
  return a.Env().Undefined();
}

Napi::Value UploadCoeff(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_upload_coeff(Ctx(a[0]), Int(a[1]), Ptr<double>(a[2]), Len<double>(a[2])), "uploadCoeff");
  return a.Env().Undefined();
}

// A face object of cpml.js:147-448 (_initFace_x/y/z): profiles b_e a_e b_m a_m
// (length nc) and the four CPsi arrays of its axis, in the slot order of
// fdtd_ctx_upload_cpml (H first, then E).
Napi::Value UploadCpml(const Napi::CallbackInfo& a) {
  Napi::Object f = a[2].As<Napi::Object>();
  static const char* const kSlots[3][4] = {{"CPsi_hyx", "CPsi_hzx", "CPsi_eyx", "CPsi_ezx"},
                                           {"CPsi_hxy", "CPsi_hzy", "CPsi_ezy", "CPsi_exy"},
                                           {"CPsi_hxz", "CPsi_hyz", "CPsi_exz", "CPsi_eyz"}};
  static const char* const kMStart[3] = {"i_m_start", "j_m_start", "k_m_start"};
  static const char* const kEStart[3] = {"i_e_start", "j_e_start", "k_e_start"};
  const int face = Int(a[1]);
  if (face < 0 || face > 5) throw Napi::Error::New(a.Env(), "uploadCpml: face id must be 0..5");
  const int axis = face / 2;
  const double* cp[4];
  long n[4];
  for (int s = 0; s < 4; s++) {
    Napi::Value v = f.Get(kSlots[axis][s]);
    cp[s] = Ptr<double>(v);
    n[s] = Len<double>(v);
  }
  Check(a.Env(),
        fdtd_ctx_upload_cpml(Ctx(a[0]), face, Int(f.Get("nc")), Ptr<double>(f.Get("b_e")), Ptr<double>(f.Get("a_e")),
                             Ptr<double>(f.Get("b_m")), Ptr<double>(f.Get("a_m")), nullptr, nullptr, cp[0], n[0],
                             cp[1], n[1], cp[2], n[2], cp[3], n[3], Int(f.Get(kMStart[axis])),
                             Int(f.Get(kEStart[axis]))),
        "uploadCpml");
  return a.Env().Undefined();
}

Napi::Value AddVSource(const Napi::CallbackInfo& a) {
  Check(a.Env(),
        fdtd_ctx_add_vsource(Ctx(a[0]), Int(a[1]), Ptr<int>(a[2]), Ptr<double>(a[3]), (int)Len<int>(a[2]),
                             Ptr<double>(a[4]), (int)Len<double>(a[4])),
        "addVSource");
  return a.Env().Undefined();
}

Napi::Value AddSVoltage(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_add_svoltage(Ctx(a[0]), Int(a[1]), Ptr<int>(a[2]), (int)Len<int>(a[2]), Dbl(a[3])),
        "addSVoltage");
  return a.Env().Undefined();
}

Napi::Value AddSCurrent(const Napi::CallbackInfo& a) {
  Check(a.Env(),
        fdtd_ctx_add_scurrent(Ctx(a[0]), Ptr<int>(a[1]), Ptr<int>(a[2]), Ptr<double>(a[3]), (int)Len<int>(a[1])),
        "addSCurrent");
  return a.Env().Undefined();
}

// The ff object of farfield.js:28-78: frequencies and the 1-based box bounds.
Napi::Value SetupFarfield(const Napi::CallbackInfo& a) {
  Napi::Object f = a[1].As<Napi::Object>();
  Napi::Array fr = f.Get("frequencies").As<Napi::Array>();
  std::vector<double> freqs(fr.Length());
  for (uint32_t q = 0; q < fr.Length(); q++) freqs[q] = Dbl(fr.Get(q));
  Check(a.Env(),
        fdtd_ctx_setup_farfield(Ctx(a[0]), (int)freqs.size(), freqs.data(), Int(f.Get("li")), Int(f.Get("lj")),
                                Int(f.Get("lk")), Int(f.Get("ui")), Int(f.Get("uj")), Int(f.Get("uk"))),
        "setupFarfield");
  return a.Env().Undefined();
}

Napi::Value Run(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_run(Ctx(a[0]), Int(a[1])), "run");
  return a.Env().Undefined();
}

Napi::Value Step(const Napi::CallbackInfo& a) { return Napi::Number::New(a.Env(), fdtd_ctx_step(Ctx(a[0]))); }

Napi::Value Status(const Napi::CallbackInfo& a) {
  int code = 0, step = -1;
  Check(a.Env(), fdtd_status(Ctx(a[0]), &code, &step), "status");
  Napi::Object o = Napi::Object::New(a.Env());
  o.Set("code", Napi::Number::New(a.Env(), code));
  o.Set("step", Napi::Number::New(a.Env(), step));
  return o;
}

Napi::Value ReadTrace(const Napi::CallbackInfo& a) {
  Check(a.Env(),
        fdtd_ctx_read_trace(Ctx(a[0]), Int(a[1]), Int(a[2]), Ptr<double>(a[3]), (int)Len<double>(a[3])),
        "readTrace");
  return a.Env().Undefined();
}

Napi::Value ReadField(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_read_field(Ctx(a[0]), Int(a[1]), Ptr<double>(a[2]), Len<double>(a[2])), "readField");
  return a.Env().Undefined();
}

Napi::Value ReadFarfield(const Napi::CallbackInfo& a) {
  Check(a.Env(),
        fdtd_ctx_read_farfield(Ctx(a[0]), Int(a[1]), Ptr<double>(a[2]), Ptr<double>(a[3]), Len<double>(a[2])),
        "readFarfield");
  return a.Env().Undefined();
}

Napi::Value FarfieldPost(const Napi::CallbackInfo& a) {
  Napi::Env env = a.Env();
  const int nang = (int)Len<double>(a[1]);
  const int nf = Int(a[3]);
  if (Len<double>(a[2]) != nang) throw Napi::Error::New(env, "farfieldPost: theta and phi lengths differ");
  Napi::Float64Array radp = Napi::Float64Array::New(env, nf > 0 ? nf : 1);
  Napi::Float64Array dth = Napi::Float64Array::New(env, (size_t)(nf > 0 ? nf : 1) * nang);
  Napi::Float64Array dph = Napi::Float64Array::New(env, (size_t)(nf > 0 ? nf : 1) * nang);
  Check(env,
        fdtd_ctx_farfield_post(Ctx(a[0]), Ptr<double>(a[1]), Ptr<double>(a[2]), nang, radp.Data(), dth.Data(),
                               dph.Data()),
        "farfieldPost");
  Napi::Object o = Napi::Object::New(env);
  o.Set("radp", radp);
  o.Set("dTheta", dth);
  o.Set("dPhi", dph);
  return o;
}

Napi::Value Dft(const Napi::CallbackInfo& a) {
  Napi::Env env = a.Env();
  const int m = (int)Len<double>(a[2]);
  Napi::Float64Array re = Napi::Float64Array::New(env, m), im = Napi::Float64Array::New(env, m);
  Check(env,
        fdtd_dft(Ptr<double>(a[0]), (int)Len<double>(a[0]), Dbl(a[1]), Ptr<double>(a[2]), m, Dbl(a[3]), re.Data(),
                 im.Data()),
        "dft");
  Napi::Object o = Napi::Object::New(env);
  o.Set("re", re);
  o.Set("im", im);
  return o;
}

Napi::Value SaveState(const Napi::CallbackInfo& a) {
  Napi::Env env = a.Env();
  long long n = 0;
  Check(env, fdtd_ctx_state_size(Ctx(a[0]), &n), "saveState");
  Napi::Buffer<unsigned char> buf = Napi::Buffer<unsigned char>::New(env, (size_t)n);
  Check(env, fdtd_ctx_save_state(Ctx(a[0]), buf.Data(), n), "saveState");
  return buf;
}

Napi::Value LoadState(const Napi::CallbackInfo& a) {
  Napi::Buffer<unsigned char> buf = a[1].As<Napi::Buffer<unsigned char>>();
  Check(a.Env(), fdtd_ctx_load_state(Ctx(a[0]), buf.Data(), (long long)buf.Length()), "loadState");
  return a.Env().Undefined();
}

Napi::Value SetDftBlock(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_set_dft_block(Ctx(a[0]), Int(a[1])), "setDftBlock");
  return a.Env().Undefined();
}

Napi::Value SetDftAccumulator(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_set_dft_accumulator(Ctx(a[0]), Int(a[1])), "setDftAccumulator");
  return a.Env().Undefined();
}

Napi::Value SetXWall(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_ctx_set_x_wall(Ctx(a[0]), Int(a[1])), "setXWall");
  return a.Env().Undefined();
}

Napi::Value BatchCreate(const Napi::CallbackInfo& a) {
  Napi::Array arr = a[0].As<Napi::Array>();
  std::vector<fdtd_ctx*> hs(arr.Length());
  for (uint32_t q = 0; q < arr.Length(); q++) hs[q] = Ctx(arr.Get(q));
  fdtd_batch* b = nullptr;
  Check(a.Env(), fdtd_batch_create(hs.data(), (int)hs.size(), &b), "batchCreate");
  return Napi::External<fdtd_batch>::New(a.Env(), b);
}

Napi::Value BatchRun(const Napi::CallbackInfo& a) {
  Check(a.Env(), fdtd_batch_run(Batch(a[0]), Int(a[1])), "batchRun");
  return a.Env().Undefined();
}

// (b, chunk, rows, prefetch, group, streams, width[, perLaunch]): a launch
// shape as the autotuner reports it (special-topics_b200/autotune.py,
// tune_batch); perLaunch > 0 selects grouped launches.
Napi::Value BatchShape(const Napi::CallbackInfo& a) {
  fdtd_batch* b = Batch(a[0]);
  Check(a.Env(), fdtd_batch_set_tiling(b, Int(a[1]), Int(a[2]), Int(a[3]), Int(a[4])), "batchShape");
  Check(a.Env(), fdtd_batch_set_streams(b, Int(a[5])), "batchShape");
  Check(a.Env(), fdtd_batch_set_block_width(b, Int(a[6])), "batchShape");
  Check(a.Env(), fdtd_batch_set_members_per_launch(b, a.Length() > 7 ? Int(a[7]) : 0), "batchShape");
  return a.Env().Undefined();
}

Napi::Value BatchFree(const Napi::CallbackInfo& a) {
  fdtd_batch_free(Batch(a[0]));
  return a.Env().Undefined();
}

Napi::Object Init(Napi::Env env, Napi::Object e) {
  e.Set("deviceCount", Napi::Function::New(env, DeviceCount));
  e.Set("create", Napi::Function::New(env, Create));
  e.Set("free", Napi::Function::New(env, Free));
  e.Set("uploadCoeff", Napi::Function::New(env, UploadCoeff));
  e.Set("uploadCpml", Napi::Function::New(env, UploadCpml));
  e.Set("addVSource", Napi::Function::New(env, AddVSource));
  e.Set("addSVoltage", Napi::Function::New(env, AddSVoltage));
  e.Set("addSCurrent", Napi::Function::New(env, AddSCurrent));
  e.Set("setupFarfield", Napi::Function::New(env, SetupFarfield));
  e.Set("run", Napi::Function::New(env, Run));
  e.Set("step", Napi::Function::New(env, Step));
  e.Set("status", Napi::Function::New(env, Status));
  e.Set("readTrace", Napi::Function::New(env, ReadTrace));
  e.Set("readField", Napi::Function::New(env, ReadField));
  e.Set("readFarfield", Napi::Function::New(env, ReadFarfield));
  e.Set("farfieldPost", Napi::Function::New(env, FarfieldPost));
  e.Set("dft", Napi::Function::New(env, Dft));
  e.Set("saveState", Napi::Function::New(env, SaveState));
  e.Set("loadState", Napi::Function::New(env, LoadState));
  e.Set("setDftBlock", Napi::Function::New(env, SetDftBlock));
  e.Set("setDftAccumulator", Napi::Function::New(env, SetDftAccumulator));
  e.Set("setXWall", Napi::Function::New(env, SetXWall));
  e.Set("batchCreate", Napi::Function::New(env, BatchCreate));
  e.Set("batchRun", Napi::Function::New(env, BatchRun));
  e.Set("batchShape", Napi::Function::New(env, BatchShape));
  e.Set("batchFree", Napi::Function::New(env, BatchFree));
  return e;
}

}  // namespace

NODE_API_MODULE(fdtd_b200, Init)
