package dev.gravity

import java.nio.FloatBuffer

/**
 * JNI bindings of include/p3m.h (the glue is gravity_p3m_jni.c beside this
 * file). Every function returns a p3m_status; [check] throws the exception
 * the reference throws for the same condition.
 *
 * Inside GravityPipeline (src/main/kotlin/dev/gravity/GravityPipeline.kt) the
 * P3M seam becomes: the constructor calls [create] (buffers :183-246, kernel
 * spectra :1341-1371), initializeAcceleration (:366-370) calls
 * [initializeAcceleration], the gravity part of step (:445-494) calls [step],
 * the `bounded` / `fieldAccelerationX/Y` / `mutualGravity` / `massExcess`
 * setters (:97-121, :213) forward to the setters below, uploadBodies
 * (:720-770) calls [uploadRange] with the direct buffers it already fills,
 * and close (:1556-1620) calls [destroy].
 */
internal object P3mNative {
    init { System.loadLibrary("gravity_p3m_jni") }

    external fun create(
        viewportWidth: Int, viewportHeight: Int, gridWidth: Int, gridHeight: Int,
        gravity: Float, softeningCells: Float, searchSigmaMultiplier: Float,
        minimumRadius: Int, maximumRadius: Int, exactLimit: Int, homeLimit: Int,
        minimumDistanceFraction: Float, windowPowerFloor: Float,
        timeStep: Float, driftSubsteps: Int, sortInterval: Int,
        capacity: Int, bounded: Boolean, int64Deposit: Boolean, mutualGravity: Boolean,
        out: LongArray,
    ): Int

    external fun destroy(ctx: Long): Int
    external fun lastError(ctx: Long): String
    external fun uploadRange(ctx: Long, first: Int, count: Int, bodies: FloatBuffer?,
                             materials: FloatBuffer?): Int
    external fun download(ctx: Long, n: Int, bodies: FloatBuffer?, acceleration: FloatBuffer?): Int
    external fun setBounded(ctx: Long, bounded: Boolean): Int
    external fun setField(ctx: Long, axPixels: Float, ayPixels: Float): Int
    external fun setMutualGravity(ctx: Long, enabled: Boolean): Int
    external fun setMassExcess(ctx: Long, excess: Float): Int
    external fun initializeAcceleration(ctx: Long, n: Int): Int
    external fun step(ctx: Long, n: Int, steps: Int): Int
    /** One step with its upload and read-back pipelined against the
     *  neighbouring steps (p3m_step_io): [bodiesIn] becomes the first [n]
     *  bodies, the stepped bodies go to [bodiesOut]. Direct buffers, left
     *  untouched until [synchronize]. */
    external fun stepIo(ctx: Long, n: Int, bodiesIn: FloatBuffer?, bodiesOut: FloatBuffer?): Int
    external fun synchronize(ctx: Long): Int

    /** p3m_status -> the reference's exceptions: invalid argument, capacity and
     *  unsupported configuration are require() failures, the rest check(). */
    fun Int.check(ctx: Long) {
        if (this == 0) return
        val message = lastError(ctx)
        if (this == -1 || this == -6 || this == -7) throw IllegalArgumentException(message)
        throw IllegalStateException(message)
    }
}
