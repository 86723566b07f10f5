/* fgkl_jni.c: fgkl's JNI entry points (crates/jni/src/lib.rs:150-313) over include/fgkl_b200.h. */
#include <jni.h>
#include <stdint.h>
#include <stdlib.h>
#include "fgkl_b200.h"

static void throw_for(JNIEnv* env, int rc) {
  if ((*env)->ExceptionCheck(env)) return;
  const char* cls = (rc >= FGKL_E_INVALID_ARGUMENT && rc <= FGKL_E_EMPTY_READ) || rc == FGKL_E_UNSUPPORTED ||
                            rc == FGKL_E_EMPTY_SEQUENCE
                        ? "java/lang/IllegalArgumentException" : "java/lang/RuntimeException";
  (*env)->ThrowNew(env, (*env)->FindClass(env, cls), fgkl_last_error());
}

/* A native allocation failed: fgkl's panic path (crates/jni/src/lib.rs:39-74) throws RuntimeException. */
static void throw_out_of_memory(JNIEnv* env) {
  if ((*env)->ExceptionCheck(env)) return;
  (*env)->ThrowNew(env, (*env)->FindClass(env, "java/lang/RuntimeException"), "native memory allocation failed");
}

/* Copies a Java byte[] into native memory; NULL when malloc fails. */
static jbyte* bytes(JNIEnv* env, jbyteArray a, jsize* n) {
  *n = (*env)->GetArrayLength(env, a);
  jbyte* p = malloc(*n ? (size_t)*n : 1);
  if (p) (*env)->GetByteArrayRegion(env, a, 0, *n, p);
  return p;
}
static jint* ints(JNIEnv* env, jintArray a, jsize* n) {
  *n = (*env)->GetArrayLength(env, a);
  jint* p = malloc(*n ? (size_t)*n * sizeof(jint) : 1);
  if (p) (*env)->GetIntArrayRegion(env, a, 0, *n, p);
  return p;
}

static void compute(JNIEnv* env, int pd, jbyteArray bases, jbyteArray quals, jbyteArray ins, jbyteArray del,
                    jbyteArray gcp, jintArray read_offsets, jbyteArray hap_bases, jbyteArray hap_flags,
                    jintArray hap_offsets, jboolean double_precision, jdoubleArray likelihoods) {
  jsize nb, nq, ni, nd, ng, nro, nhb, nhf = 0, nho;
  jbyte *b = bytes(env, bases, &nb), *q = bytes(env, quals, &nq), *i = bytes(env, ins, &ni),
        *d = bytes(env, del, &nd), *g = bytes(env, gcp, &ng), *hb = bytes(env, hap_bases, &nhb),
        *hf = pd ? bytes(env, hap_flags, &nhf) : NULL;
  jint *ro = ints(env, read_offsets, &nro), *ho = ints(env, hap_offsets, &nho);
  double* out = NULL;
  jsize n_out = 0;
  if (!(*env)->ExceptionCheck(env)) {
    n_out = (*env)->GetArrayLength(env, likelihoods);
    out = malloc(n_out ? (size_t)n_out * sizeof(double) : 1);
    if (!b || !q || !i || !d || !g || !hb || (pd && !hf) || !ro || !ho || !out) throw_out_of_memory(env);
  }
  if (!(*env)->ExceptionCheck(env)) {
    fgkl_reads r = {(const uint8_t*)b, nb, (const uint8_t*)q, nq, (const uint8_t*)i, ni,
                    (const uint8_t*)d, nd, (const uint8_t*)g, ng, ro, nro};
    fgkl_haplotypes h = {(const uint8_t*)hb, nhb, (const uint8_t*)hf, nhf, ho, nho};
    const int rc = pd ? fgkl_pdhmm_compute(&r, &h, double_precision ? 1 : 0, out, n_out)
                      : fgkl_pairhmm_compute(&r, &h, double_precision ? 1 : 0, out, n_out);
    if (rc != FGKL_OK) throw_for(env, rc);
    else (*env)->SetDoubleArrayRegion(env, likelihoods, 0, n_out, out);
  }
  free(b); free(q); free(i); free(d); free(g); free(hb); free(hf); free(ro); free(ho); free(out);
}

JNIEXPORT void JNICALL Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_computeNative(
    JNIEnv* env, jclass cls, jbyteArray bases, jbyteArray quals, jbyteArray ins_gop, jbyteArray del_gop,
    jbyteArray gcp, jintArray read_offsets, jbyteArray hap_bases, jintArray hap_offsets,
    jboolean double_precision, jdoubleArray likelihoods) {
  (void)cls;
  compute(env, 0, bases, quals, ins_gop, del_gop, gcp, read_offsets, hap_bases, NULL, hap_offsets,
          double_precision, likelihoods);
}

JNIEXPORT void JNICALL Java_com_fulcrumgenomics_fgkl_pdhmm_FgklPdHmm_computeNative(
    JNIEnv* env, jclass cls, jbyteArray bases, jbyteArray quals, jbyteArray ins_gop, jbyteArray del_gop,
    jbyteArray gcp, jintArray read_offsets, jbyteArray hap_bases, jbyteArray hap_flags, jintArray hap_offsets,
    jboolean double_precision, jdoubleArray likelihoods) {
  (void)cls;
  compute(env, 1, bases, quals, ins_gop, del_gop, gcp, read_offsets, hap_bases, hap_flags, hap_offsets,
          double_precision, likelihoods);
}

JNIEXPORT jobject JNICALL Java_com_fulcrumgenomics_fgkl_pairhmm_FgklPairHmm_backendNative(JNIEnv* env, jclass c) {
  (void)c;
  return (*env)->NewStringUTF(env, fgkl_backend());
}
JNIEXPORT jobject JNICALL Java_com_fulcrumgenomics_fgkl_pdhmm_FgklPdHmm_backendNative(JNIEnv* env, jclass c) {
  (void)c;
  return (*env)->NewStringUTF(env, fgkl_backend());
}

/* FgklSmithWaterman.alignNative (crates/jni/src/lib.rs:271-313): the CIGAR string, with the
 * alignment offset written to offset[0]. */
JNIEXPORT jobject JNICALL Java_com_fulcrumgenomics_fgkl_smithwaterman_FgklSmithWaterman_alignNative(
    JNIEnv* env, jclass cls, jbyteArray reference, jbyteArray alternate, jint match_value, jint mismatch_penalty,
    jint gap_open, jint gap_extend, jint strategy, jintArray offset) {
  (void)cls;
  jsize nr, na;
  jbyte *r = bytes(env, reference, &nr), *a = bytes(env, alternate, &na);
  const size_t cap = 16 * ((size_t)nr + (size_t)na + 4);
  char* cigar = NULL;
  jobject result = NULL;
  if (!(*env)->ExceptionCheck(env)) {
    cigar = malloc(cap);
    if (!r || !a || !cigar) throw_out_of_memory(env);
  }
  if (!(*env)->ExceptionCheck(env)) {
    const fgkl_sw_params p = {match_value, mismatch_penalty, gap_open, gap_extend};
    int32_t off = 0;
    const int rc = fgkl_sw_align((const uint8_t*)r, nr, (const uint8_t*)a, na, &p, strategy, cigar, (int64_t)cap, &off);
    if (rc != FGKL_OK) {
      throw_for(env, rc);
    } else {
      (*env)->SetIntArrayRegion(env, offset, 0, 1, &off);
      result = (*env)->NewStringUTF(env, cigar);
    }
  }
  free(r); free(a); free(cigar);
  return result;
}

JNIEXPORT jobject JNICALL Java_com_fulcrumgenomics_fgkl_smithwaterman_FgklSmithWaterman_backendNative(JNIEnv* env, jclass c) {
  (void)c;
  return (*env)->NewStringUTF(env, fgkl_backend());
}
