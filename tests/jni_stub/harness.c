/* A fake JNI environment over plain C arrays, driving fgkl_b200/jni/fgkl_jni.c's entry points as a
 * JVM would (test infrastructure only): Java arrays become fake objects holding a length and a copy
 * of the data, exceptions are recorded as (class, message), and the shim's output array is read
 * back after the call. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "jni.h"

struct fake_object {
  int kind; /* 1 byte[], 2 int[], 3 double[], 4 class, 5 string */
  jsize len;
  void* data;
  char name[2048];
};

typedef struct {
  int thrown;
  char cls[128];
  char msg[512];
  int region_calls; /* SetDoubleArrayRegion calls */
  struct fake_object classes[4];
  int n_classes;
  struct fake_object str;
} fake_state;

static fake_state* state(JNIEnv* env) { return (fake_state*)(*env)->context; }
static jboolean exception_check(JNIEnv* env) { return (jboolean)(state(env)->thrown != 0); }
static jint throw_new(JNIEnv* env, jclass cls, const char* msg) {
  fake_state* s = state(env);
  s->thrown = 1;
  snprintf(s->cls, sizeof s->cls, "%.127s", cls ? cls->name : "");
  snprintf(s->msg, sizeof s->msg, "%s", msg ? msg : "");
  return 0;
}
static jclass find_class(JNIEnv* env, const char* name) {
  fake_state* s = state(env);
  struct fake_object* c = &s->classes[s->n_classes++ % 4];
  c->kind = 4;
  snprintf(c->name, sizeof c->name, "%s", name);
  return c;
}
static jsize array_length(JNIEnv* env, jarray a) { (void)env; return a ? a->len : 0; }
static void get_bytes(JNIEnv* env, jbyteArray a, jsize start, jsize len, jbyte* buf) {
  (void)env;
  if (len > 0) memcpy(buf, (const jbyte*)a->data + start, (size_t)len);
}
static void get_ints(JNIEnv* env, jintArray a, jsize start, jsize len, jint* buf) {
  (void)env;
  if (len > 0) memcpy(buf, (const jint*)a->data + start, (size_t)len * sizeof(jint));
}
static void set_doubles(JNIEnv* env, jdoubleArray a, jsize start, jsize len, const jdouble* buf) {
  state(env)->region_calls++;
  if (len > 0) memcpy((jdouble*)a->data + start, buf, (size_t)len * sizeof(jdouble));
}
static void set_ints(JNIEnv* env, jintArray a, jsize start, jsize len, const jint* buf) {
  (void)env;
  if (len > 0) memcpy((jint*)a->data + start, buf, (size_t)len * sizeof(jint));
}
static jstring new_string(JNIEnv* env, const char* utf) {
  fake_state* s = state(env);
  s->str.kind = 5;
  snprintf(s->str.name, sizeof s->str.name, "%s", utf);
  return &s->str;
}

/* The shim's entry points (fgkl_jni.c). */
void Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_computeNative(JNIEnv*, jclass, jbyteArray, jbyteArray, jbyteArray,
                                                                    jbyteArray, jbyteArray, jintArray, jbyteArray,
                                                                    jintArray, jboolean, jdoubleArray);
void Java_com_fulcrumgenomics_fgkl_pdhmm_FgklPdHmm_computeNative(JNIEnv*, jclass, jbyteArray, jbyteArray, jbyteArray,
                                                                jbyteArray, jbyteArray, jintArray, jbyteArray, jbyteArray,
                                                                jintArray, jboolean, jdoubleArray);
jobject Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_backendNative(JNIEnv*, jclass);
jobject Java_com_fulcrumgenomics_fgkl_smithwaterman_FgklSmithWaterman_alignNative(JNIEnv*, jclass, jbyteArray, jbyteArray, jint,
                                                                                  jint, jint, jint, jint, jintArray);

static struct fake_object arr(int kind, const void* data, jsize len) {
  struct fake_object o;
  memset(&o, 0, sizeof o);
  o.kind = kind;
  o.len = len;
  o.data = (void*)data;
  return o;
}

/* Calls computeNative (PD when hap_flags is not NULL) with Java arrays holding the given data.
 * Returns 1 if the shim threw (class and message copied out), else 0 with `out` filled through
 * SetDoubleArrayRegion; *region_calls counts those calls. */
int harness_compute(const int8_t* bases, int nb, const int8_t* quals, int nq, const int8_t* ins, int ni,
                    const int8_t* del, int nd, const int8_t* gcp, int ng, const int32_t* roff, int nro,
                    const int8_t* hap_bases, int nhb, const int8_t* hap_flags, int nhf, const int32_t* hoff, int nho,
                    int double_precision, double* out, int n_out, char* cls, char* msg, int* region_calls) {
  fake_state s;
  memset(&s, 0, sizeof s);
  struct JNINativeInterface_ fns = {&s, exception_check, throw_new, find_class, array_length,
                                    get_bytes, get_ints, set_doubles, new_string, set_ints};
  JNIEnv env = &fns;
  struct fake_object b = arr(1, bases, nb), q = arr(1, quals, nq), i = arr(1, ins, ni), d = arr(1, del, nd),
                     g = arr(1, gcp, ng), ro = arr(2, roff, nro), hb = arr(1, hap_bases, nhb), hf = arr(1, hap_flags, nhf),
                     ho = arr(2, hoff, nho), o = arr(3, out, n_out);
  if (hap_flags)
    Java_com_fulcrumgenomics_fgkl_pdhmm_FgklPdHmm_computeNative(&env, NULL, &b, &q, &i, &d, &g, &ro, &hb, &hf, &ho,
                                                               (jboolean)(double_precision != 0), &o);
  else
    Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_computeNative(&env, NULL, &b, &q, &i, &d, &g, &ro, &hb, &ho,
                                                                   (jboolean)(double_precision != 0), &o);
  strcpy(cls, s.cls);
  strcpy(msg, s.msg);
  *region_calls = s.region_calls;
  return s.thrown;
}

/* backendNative's string. */
void harness_backend(char* out, int cap) {
  fake_state s;
  memset(&s, 0, sizeof s);
  struct JNINativeInterface_ fns = {&s, exception_check, throw_new, find_class, array_length,
                                    get_bytes, get_ints, set_doubles, new_string, set_ints};
  JNIEnv env = &fns;
  jobject str = Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_backendNative(&env, NULL);
  snprintf(out, (size_t)cap, "%s", str ? str->name : "");
}

/* Calls FgklSmithWaterman.alignNative; returns 1 if it threw (class and message copied out), else 0
 * with the CIGAR string in `cigar` and the offset in *offset. */
int harness_sw_align(const int8_t* ref, int nr, const int8_t* alt, int na, int match, int mismatch, int open, int extend,
                     int strategy, char* cigar, int cap, int32_t* offset, char* cls, char* msg) {
  fake_state s;
  memset(&s, 0, sizeof s);
  struct JNINativeInterface_ fns = {&s, exception_check, throw_new, find_class, array_length,
                                    get_bytes, get_ints, set_doubles, new_string, set_ints};
  JNIEnv env = &fns;
  int32_t off[1] = {-1};
  struct fake_object r = arr(1, ref, nr), a = arr(1, alt, na), o = arr(2, off, 1);
  jobject str = Java_com_fulcrumgenomics_fgkl_smithwaterman_FgklSmithWaterman_alignNative(&env, NULL, &r, &a, match, mismatch,
                                                                                          open, extend, strategy, &o);
  snprintf(cigar, (size_t)cap, "%s", str ? str->name : "");
  *offset = off[0];
  strcpy(cls, s.cls);
  strcpy(msg, s.msg);
  return s.thrown;
}
