// Stand-in for node-addon-api's napi.h, for compile checks only.
//
// Neither Node.js nor node_api.h is available here, so the real header cannot
// be used.  This declares just the part of the Napi C++ API that
// integration/node/binding_b200.cpp uses, with the same names and call
// shapes, so that `g++ -fsyntax-only` type-checks the binding's calls into
// include/fdtd_b200.h.  Nothing here runs.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

namespace Napi {

class Env;
class Value;

class Env {
 public:
  Value Undefined() const;
};

class Value {
 public:
  template <class T>
  T As() const;
};

class Number : public Value {
 public:
  static Number New(Env, double);
  int32_t Int32Value() const;
  double DoubleValue() const;
};

class Object : public Value {
 public:
  static Object New(Env);
  Value Get(const char*) const;
  bool Has(const char*) const;
  void Set(const char*, const Value&);
};

class Array : public Object {
 public:
  uint32_t Length() const;
  Value Get(uint32_t) const;
};

template <class T>
class External : public Value {
 public:
  static External New(Env, T*);
  T* Data() const;
};

template <class T>
class TypedArrayOf : public Value {
 public:
  static TypedArrayOf New(Env, size_t);
  T* Data() const;
  size_t ElementLength() const;
};
using Float64Array = TypedArrayOf<double>;
using Int32Array = TypedArrayOf<int32_t>;

template <class T>
class Buffer : public Value {
 public:
  static Buffer New(Env, size_t);
  T* Data() const;
  size_t Length() const;
};

class CallbackInfo {
 public:
  Value operator[](size_t) const;
  Napi::Env Env() const;
  size_t Length() const;
};

class Function : public Value {
 public:
  static Function New(Env, Value (*)(const CallbackInfo&));
};

class Error {
 public:
  static Error New(Env, const std::string&);
};

}  // namespace Napi

#define NODE_API_MODULE(name, init) \
  static Napi::Object (*napi_module_init_##name)(Napi::Env, Napi::Object) = init;
