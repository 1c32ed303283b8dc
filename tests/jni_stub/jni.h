/*
 * A minimal stand-in for a JDK's <jni.h>: the JNI types and the three
 * JNIEnv functions gravity_b200/jni/gravity_p3m_jni.c uses, with the names
 * and signatures of the JNI specification. Test infrastructure only: it lets
 * the CPU tests compile the glue and call it through a fake environment
 * (harness.c) where no JDK is installed.
 */
#ifndef GRAVITY_TEST_JNI_STUB_H
#define GRAVITY_TEST_JNI_STUB_H

#include <stdint.h>

#define JNIEXPORT __attribute__((visibility("default")))
#define JNICALL

typedef int32_t jint;
typedef int64_t jlong;
typedef float jfloat;
typedef uint8_t jboolean;
typedef jint jsize;
typedef void* jobject;
typedef jobject jclass;
typedef jobject jstring;
typedef jobject jarray;
typedef jarray jlongArray;

struct JNINativeInterface_;
typedef const struct JNINativeInterface_* JNIEnv;

struct JNINativeInterface_ {
    jstring (*NewStringUTF)(JNIEnv* env, const char* utf);
    void (*SetLongArrayRegion)(JNIEnv* env, jlongArray array, jsize start, jsize len,
                               const jlong* buf);
    void* (*GetDirectBufferAddress)(JNIEnv* env, jobject buf);
};

#endif
