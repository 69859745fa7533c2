// The slice of the Java Native Interface the JNI shim (jni_bridge.cpp) needs,
// written from the JNI specification: the primitive types, and JNIEnv as a
// pointer to the JVM's function table, whose entries sit at the indices the
// specification's "Interface Function Table" assigns (the first four are
// reserved). The table layout is fixed by the specification, so a library
// built against this header binds to any JVM; no JDK is needed to build it.
#pragma once

#include <cstdint>

#if defined(_WIN32)
#define AERO_JNIEXPORT __declspec(dllexport)
#define AERO_JNICALL __stdcall
#else
#define AERO_JNIEXPORT __attribute__((visibility("default")))
#define AERO_JNICALL
#endif

namespace aero_jni {

typedef uint8_t jboolean;
typedef int8_t jbyte;
typedef uint16_t jchar;
typedef int16_t jshort;
typedef int32_t jint;
typedef int64_t jlong;
typedef float jfloat;
typedef double jdouble;
typedef jint jsize;

struct Object;
typedef Object* jobject;
typedef jobject jclass;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jbyteArray;
typedef jarray jshortArray;
typedef jarray jintArray;
typedef jarray jfloatArray;

constexpr jboolean JNI_FALSE = 0;
constexpr jboolean JNI_TRUE = 1;
constexpr jint JNI_COMMIT = 1;  // Release*ArrayElements: copy back, keep the buffer
constexpr jint JNI_ABORT = 2;   // Release*ArrayElements: free the buffer, no copy back

// Function table indices (JNI specification, "Interface Function Table").
enum Slot : int {
    kNewStringUTF = 167,
    kGetArrayLength = 171,
    kNewIntArray = 179,
    kNewFloatArray = 181,
    kGetByteArrayElements = 184,
    kGetShortArrayElements = 186,
    kGetIntArrayElements = 187,
    kGetFloatArrayElements = 189,
    kReleaseByteArrayElements = 192,
    kReleaseShortArrayElements = 194,
    kReleaseIntArrayElements = 195,
    kReleaseFloatArrayElements = 197,
    kSetIntArrayRegion = 211,
    kSetFloatArrayRegion = 213,
    kTableSize = 235
};

struct FunctionTable {
    void* slot[kTableSize];
};
// JNIEnv: what the JVM passes as the first argument of every native method.
typedef const FunctionTable* JNIEnv;

template <typename F>
inline F fn(JNIEnv* env, Slot s) {
    return reinterpret_cast<F>((*env)->slot[s]);
}

inline jsize array_length(JNIEnv* env, jarray a) {
    return fn<jsize(AERO_JNICALL*)(JNIEnv*, jarray)>(env, kGetArrayLength)(env, a);
}
inline jstring new_string_utf(JNIEnv* env, const char* s) {
    return fn<jstring(AERO_JNICALL*)(JNIEnv*, const char*)>(env, kNewStringUTF)(env, s);
}
inline jintArray new_int_array(JNIEnv* env, jsize n) {
    return fn<jintArray(AERO_JNICALL*)(JNIEnv*, jsize)>(env, kNewIntArray)(env, n);
}
inline jfloatArray new_float_array(JNIEnv* env, jsize n) {
    return fn<jfloatArray(AERO_JNICALL*)(JNIEnv*, jsize)>(env, kNewFloatArray)(env, n);
}
inline void set_int_region(JNIEnv* env, jintArray a, jsize start, jsize n, const jint* v) {
    fn<void(AERO_JNICALL*)(JNIEnv*, jintArray, jsize, jsize, const jint*)>(env, kSetIntArrayRegion)(env, a, start, n, v);
}
inline void set_float_region(JNIEnv* env, jfloatArray a, jsize start, jsize n, const jfloat* v) {
    fn<void(AERO_JNICALL*)(JNIEnv*, jfloatArray, jsize, jsize, const jfloat*)>(env, kSetFloatArrayRegion)(env, a, start, n, v);
}

// Get<T>ArrayElements / Release<T>ArrayElements slots per element type.
template <typename T> struct ElementSlots;
template <> struct ElementSlots<jbyte> { static constexpr Slot get = kGetByteArrayElements, release = kReleaseByteArrayElements; };
template <> struct ElementSlots<jshort> { static constexpr Slot get = kGetShortArrayElements, release = kReleaseShortArrayElements; };
template <> struct ElementSlots<jint> { static constexpr Slot get = kGetIntArrayElements, release = kReleaseIntArrayElements; };
template <> struct ElementSlots<jfloat> { static constexpr Slot get = kGetFloatArrayElements, release = kReleaseFloatArrayElements; };

// The elements of a Java array for the duration of one native call. Inputs
// are released with JNI_ABORT (nothing to copy back); an output commits its
// contents (mode 0) only when commit() was called, as the reference's
// forwarders release outputs with `ok ? 0 : JNI_ABORT`.
template <typename T>
class Elements {
public:
    Elements(JNIEnv* env, jarray a) : env_(env), a_(a) {
        if (a) p_ = fn<T*(AERO_JNICALL*)(JNIEnv*, jarray, jboolean*)>(env, ElementSlots<T>::get)(env, a, nullptr);
    }
    ~Elements() {
        if (p_) fn<void(AERO_JNICALL*)(JNIEnv*, jarray, T*, jint)>(env_, ElementSlots<T>::release)(env_, a_, p_, mode_);
    }
    Elements(const Elements&) = delete;
    Elements& operator=(const Elements&) = delete;
    T* get() const { return p_; }
    explicit operator bool() const { return p_ != nullptr; }
    void commit(bool ok) { mode_ = ok ? 0 : JNI_ABORT; }

private:
    JNIEnv* env_;
    jarray a_;
    T* p_ = nullptr;
    jint mode_ = JNI_ABORT;
};

}  // namespace aero_jni
