/*
 * Minimal stand-in for a JDK's <jni.h>, used only to compile the reference
 * library's CPU path for the oracle. It declares the JNI scalar/array types
 * and a JNIEnv whose methods exist so the reference's JNI exports compile;
 * they are never called (the oracle drives the library through its plain
 * C ABI with ctypes). Every method aborts if it is ever reached.
 */
#ifndef ORACLE_JNI_STUB_H
#define ORACLE_JNI_STUB_H

#include <cstddef>
#include <cstdint>
#include <cstdlib>

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL
#define JNI_FALSE 0
#define JNI_TRUE 1
#define JNI_ABORT 2
#define JNI_COMMIT 1
#define JNI_OK 0
#define JNI_VERSION_1_8 0x00010008

typedef int32_t jint;
typedef int64_t jlong;
typedef int8_t jbyte;
typedef uint8_t jboolean;
typedef uint16_t jchar;
typedef int16_t jshort;
typedef float jfloat;
typedef double jdouble;
typedef jint jsize;

struct stub_jobject_ {};
typedef stub_jobject_* jobject;
typedef jobject jclass;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jbyteArray;
typedef jarray jshortArray;
typedef jarray jintArray;
typedef jarray jlongArray;
typedef jarray jfloatArray;
typedef jarray jdoubleArray;
typedef jarray jbooleanArray;

struct JNIEnv {
    [[noreturn]] static void unreachable() { std::abort(); }
    template <typename... A> jsize GetArrayLength(A...) { unreachable(); }
    template <typename... A> jbyte* GetByteArrayElements(A...) { unreachable(); }
    template <typename... A> jshort* GetShortArrayElements(A...) { unreachable(); }
    template <typename... A> jint* GetIntArrayElements(A...) { unreachable(); }
    template <typename... A> jlong* GetLongArrayElements(A...) { unreachable(); }
    template <typename... A> jfloat* GetFloatArrayElements(A...) { unreachable(); }
    template <typename... A> void ReleaseByteArrayElements(A...) { unreachable(); }
    template <typename... A> void ReleaseShortArrayElements(A...) { unreachable(); }
    template <typename... A> void ReleaseIntArrayElements(A...) { unreachable(); }
    template <typename... A> void ReleaseLongArrayElements(A...) { unreachable(); }
    template <typename... A> void ReleaseFloatArrayElements(A...) { unreachable(); }
    template <typename... A> void GetByteArrayRegion(A...) { unreachable(); }
    template <typename... A> void SetByteArrayRegion(A...) { unreachable(); }
    template <typename... A> void SetFloatArrayRegion(A...) { unreachable(); }
    template <typename... A> void SetIntArrayRegion(A...) { unreachable(); }
    template <typename... A> jbyteArray NewByteArray(A...) { unreachable(); }
    template <typename... A> jfloatArray NewFloatArray(A...) { unreachable(); }
    template <typename... A> jintArray NewIntArray(A...) { unreachable(); }
    template <typename... A> jstring NewStringUTF(A...) { unreachable(); }
    template <typename... A> void* GetDirectBufferAddress(A...) { unreachable(); }
    template <typename... A> jlong GetDirectBufferCapacity(A...) { unreachable(); }
    template <typename... A> jboolean ExceptionCheck(A...) { unreachable(); }
};

#endif
