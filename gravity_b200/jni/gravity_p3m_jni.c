/*
 * gravity_p3m_jni.c — JNI glue between Gravity's Kotlin GravityPipeline and
 * the C-ABI of include/p3m.h (libgravity_p3m.so).
 *
 * The reference builds with a JDK 18 toolchain (build.gradle.kts:39-41),
 * whose foreign-function API is still incubating, so the binding is JNI: the
 * `external` functions of dev.gravity.P3mNative (P3mNative.kt beside this
 * file) land here. Each forwards to one p3m_* call and returns its status;
 * the Kotlin side turns a non-zero status into the exception the reference
 * throws (require -> IllegalArgumentException, check -> IllegalStateException).
 *
 * Build (see the Makefile beside this file):
 *   cc -O2 -shared -fPIC -I$JAVA_HOME/include -I$JAVA_HOME/include/linux \
 *      -Iinclude gravity_p3m_jni.c -Lgravity_b200/lib -lgravity_p3m \
 *      -o libgravity_p3m_jni.so
 *
 * Body, material and acceleration buffers are direct NIO FloatBuffers (what
 * LWJGL's memAllocFloat returns, GravityPipeline.kt:1438-1481), passed by
 * address without a copy; a null buffer leaves that array untouched.
 */
#include <jni.h>
#include <stdint.h>

#include "p3m.h"

#define CTX(h) ((p3m_ctx*)(intptr_t)(h))
#define FN(name) Java_dev_gravity_P3mNative_##name

static float* direct(JNIEnv* env, jobject buffer) {
    return buffer ? (float*)(*env)->GetDirectBufferAddress(env, buffer) : NULL;
}

/* GravityPipeline's constructor (GravityPipeline.kt:183-246, :1341-1371):
 * GravityFieldConfig, CollisionConfig and ParticleConfig fields in the order
 * of p3m_config; the context handle is written to out[0]. */
JNIEXPORT jint JNICALL FN(create)(JNIEnv* env, jclass cls, jint viewport_width,
                                  jint viewport_height, jint grid_width, jint grid_height,
                                  jfloat gravity, jfloat softening_cells, jfloat sigma_multiplier,
                                  jint minimum_radius, jint maximum_radius, jint exact_limit,
                                  jint home_limit, jfloat minimum_distance_fraction,
                                  jfloat window_power_floor, jfloat time_step,
                                  jint drift_substeps, jint sort_interval, jint capacity,
                                  jboolean bounded, jboolean int64_deposit,
                                  jboolean mutual_gravity, jlongArray out) {
    (void)cls;
    p3m_config c;
    p3m_config_default(&c);
    c.viewport_width = viewport_width;
    c.viewport_height = viewport_height;
    c.grid_width = grid_width;
    c.grid_height = grid_height;
    c.gravitational_constant = gravity;
    c.softening_cells = softening_cells;
    c.local_search_sigma_multiplier = sigma_multiplier;
    c.minimum_neighbor_radius_cells = minimum_radius;
    c.maximum_neighbor_radius_cells = maximum_radius;
    c.exact_neighbor_body_limit = exact_limit;
    c.maximum_home_body_interactions = home_limit;
    c.minimum_distance_cell_fraction = minimum_distance_fraction;
    c.minimum_assignment_window_power = window_power_floor;
    c.time_step = time_step;
    c.drift_substeps = drift_substeps;
    c.spatial_sort_interval = sort_interval;
    c.capacity = capacity;
    c.bounded = bounded ? 1 : 0;
    c.deposit_mode = int64_deposit ? P3M_DEPOSIT_I64 : P3M_DEPOSIT_U32;
    c.mutual_gravity = mutual_gravity ? 1 : 0;
    p3m_ctx* ctx = NULL;
    const int status = p3m_create(&c, &ctx);
    const jlong handle = (jlong)(intptr_t)ctx;
    (*env)->SetLongArrayRegion(env, out, 0, 1, &handle);
    return status;
}

/* GravityPipeline.close (GravityPipeline.kt:1556-1620). */
JNIEXPORT jint JNICALL FN(destroy)(JNIEnv* env, jclass cls, jlong h) {
    (void)env; (void)cls;
    return p3m_destroy(CTX(h));
}

/* The message of the last failing call (0: of the last failing create). */
JNIEXPORT jstring JNICALL FN(lastError)(JNIEnv* env, jclass cls, jlong h) {
    (void)cls;
    return (*env)->NewStringUTF(env, p3m_last_error(CTX(h)));
}

/* seedBodies / uploadBodies (GravityPipeline.kt:720-770, :1438-1481). */
JNIEXPORT jint JNICALL FN(uploadRange)(JNIEnv* env, jclass cls, jlong h, jint first, jint count,
                                       jobject bodies, jobject materials) {
    (void)cls;
    return p3m_upload_range(CTX(h), first, count, direct(env, bodies), direct(env, materials),
                            NULL);
}

/* The SSBO readbacks (GravityPipeline.kt:378-443). */
JNIEXPORT jint JNICALL FN(download)(JNIEnv* env, jclass cls, jlong h, jint n, jobject bodies,
                                    jobject acceleration) {
    (void)cls;
    return p3m_download_state(CTX(h), direct(env, bodies), NULL, direct(env, acceleration), n);
}

/* The properties (GravityPipeline.kt:97-121, :213). */
JNIEXPORT jint JNICALL FN(setBounded)(JNIEnv* env, jclass cls, jlong h, jboolean bounded) {
    (void)env; (void)cls;
    return p3m_set_bounded(CTX(h), bounded ? 1 : 0);
}
JNIEXPORT jint JNICALL FN(setField)(JNIEnv* env, jclass cls, jlong h, jfloat ax_px, jfloat ay_px) {
    (void)env; (void)cls;
    return p3m_set_field_acceleration(CTX(h), ax_px, ay_px);
}
JNIEXPORT jint JNICALL FN(setMutualGravity)(JNIEnv* env, jclass cls, jlong h, jboolean on) {
    (void)env; (void)cls;
    return p3m_set_mutual_gravity(CTX(h), on ? 1 : 0);
}
JNIEXPORT jint JNICALL FN(setMassExcess)(JNIEnv* env, jclass cls, jlong h, jfloat excess) {
    (void)env; (void)cls;
    return p3m_set_mass_excess(CTX(h), excess);
}

/* initializeAcceleration (GravityPipeline.kt:366-370) and step
 * (GravityPipeline.kt:445-494, gravity only). */
JNIEXPORT jint JNICALL FN(initializeAcceleration)(JNIEnv* env, jclass cls, jlong h, jint n) {
    (void)env; (void)cls;
    return p3m_initialize_acceleration(CTX(h), n);
}
JNIEXPORT jint JNICALL FN(step)(JNIEnv* env, jclass cls, jlong h, jint n, jint steps) {
    (void)env; (void)cls;
    return p3m_step(CTX(h), n, steps);
}

/* A frame's upload, step and read-back with the copies pipelined against the
 * neighbouring frames (uploadBodies :720-770, step, the readback :378-443):
 * both buffers must be direct and stay untouched until synchronize. */
JNIEXPORT jint JNICALL FN(stepIo)(JNIEnv* env, jclass cls, jlong h, jint n, jobject bodies_in,
                                  jobject bodies_out) {
    (void)cls;
    return p3m_step_io(CTX(h), n, direct(env, bodies_in), direct(env, bodies_out));
}

/* Waits for the context's work; reports device-detected failures. */
JNIEXPORT jint JNICALL FN(synchronize)(JNIEnv* env, jclass cls, jlong h) {
    (void)env; (void)cls;
    return p3m_synchronize(CTX(h));
}
