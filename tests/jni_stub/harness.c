/*
 * A fake JNI environment for the CPU test of the JNI glue: jlongArray is a
 * jlong*, a direct buffer is its own address, and a jstring is the UTF-8
 * pointer handed to NewStringUTF. The harness_* functions call the glue's
 * Java_dev_gravity_P3mNative_* entry points the way the JVM would.
 */
#include <string.h>

#include <jni.h>

static jstring new_string_utf(JNIEnv* env, const char* utf) { (void)env; return (jstring)utf; }
static void set_long_array_region(JNIEnv* env, jlongArray array, jsize start, jsize len,
                                  const jlong* buf) {
    (void)env;
    memcpy((jlong*)array + start, buf, (size_t)len * sizeof(jlong));
}
static void* get_direct_buffer_address(JNIEnv* env, jobject buf) { (void)env; return buf; }

static const struct JNINativeInterface_ table = {new_string_utf, set_long_array_region,
                                                 get_direct_buffer_address};
static JNIEnv env = &table;

jint Java_dev_gravity_P3mNative_create(JNIEnv*, jclass, jint, jint, jint, jint, jfloat, jfloat,
                                       jfloat, jint, jint, jint, jint, jfloat, jfloat, jfloat,
                                       jint, jint, jint, jboolean, jboolean, jboolean, jlongArray);
jint Java_dev_gravity_P3mNative_destroy(JNIEnv*, jclass, jlong);
jstring Java_dev_gravity_P3mNative_lastError(JNIEnv*, jclass, jlong);
jint Java_dev_gravity_P3mNative_download(JNIEnv*, jclass, jlong, jint, jobject, jobject);
jint Java_dev_gravity_P3mNative_step(JNIEnv*, jclass, jlong, jint, jint);
jint Java_dev_gravity_P3mNative_stepIo(JNIEnv*, jclass, jlong, jint, jobject, jobject);

/* GravityFieldConfig defaults (GravityConfig.kt:641-654) with the given grid. */
int harness_create(int grid_width, int grid_height, long long* handle, char* message, int cap) {
    jlong out[1] = {-1};
    const jint status = Java_dev_gravity_P3mNative_create(
        &env, NULL, 2560, 1440, grid_width, grid_height, 0.035f, 0.85f, 3.0f, 1, 6, 2, 8, 0.05f,
        0.08f, 1.0f / 120.0f, 16, 2, 1000, 0, 0, 1, (jlongArray)out);
    *handle = (long long)out[0];
    const char* m = (const char*)Java_dev_gravity_P3mNative_lastError(&env, NULL, out[0]);
    strncpy(message, m ? m : "", (size_t)cap - 1);
    message[cap - 1] = '\0';
    return status;
}

int harness_destroy(long long handle) { return Java_dev_gravity_P3mNative_destroy(&env, NULL, handle); }

int harness_download(long long handle, int n, float* bodies) {
    return Java_dev_gravity_P3mNative_download(&env, NULL, handle, n, bodies, NULL);
}

int harness_step(long long handle, int n, int steps) {
    return Java_dev_gravity_P3mNative_step(&env, NULL, handle, n, steps);
}

int harness_step_io(long long handle, int n, float* bodies_in, float* bodies_out) {
    return Java_dev_gravity_P3mNative_stepIo(&env, NULL, handle, n, bodies_in, bodies_out);
}
