/* A minimal stand-in for <jni.h>, for compiling and exercising fgkl_b200/jni/fgkl_jni.c without a
 * JDK (test infrastructure only). It declares only the JNI types and the JNIEnv functions the shim
 * calls, with their JNI meanings; its function table is NOT laid out like a real JVM's, so a library
 * built against it is for the fake environment of harness.c alone, never for a JVM. */
#ifndef FGKL_TEST_JNI_STUB_H
#define FGKL_TEST_JNI_STUB_H
#include <stdint.h>

typedef int32_t jint;
typedef int64_t jlong;
typedef int8_t jbyte;
typedef uint8_t jboolean;
typedef double jdouble;
typedef jint jsize;
typedef struct fake_object* jobject;
typedef jobject jclass;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jbyteArray;
typedef jarray jintArray;
typedef jarray jdoubleArray;

struct JNINativeInterface_;
typedef const struct JNINativeInterface_* JNIEnv;

struct JNINativeInterface_ {
  void* context; /* the harness's state */
  jboolean (*ExceptionCheck)(JNIEnv* env);
  jint (*ThrowNew)(JNIEnv* env, jclass cls, const char* msg);
  jclass (*FindClass)(JNIEnv* env, const char* name);
  jsize (*GetArrayLength)(JNIEnv* env, jarray a);
  void (*GetByteArrayRegion)(JNIEnv* env, jbyteArray a, jsize start, jsize len, jbyte* buf);
  void (*GetIntArrayRegion)(JNIEnv* env, jintArray a, jsize start, jsize len, jint* buf);
  void (*SetDoubleArrayRegion)(JNIEnv* env, jdoubleArray a, jsize start, jsize len, const jdouble* buf);
  jstring (*NewStringUTF)(JNIEnv* env, const char* utf);
  void (*SetIntArrayRegion)(JNIEnv* env, jintArray a, jsize start, jsize len, const jint* buf);
};

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL
#define JNI_TRUE 1
#define JNI_FALSE 0
#endif
