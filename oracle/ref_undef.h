/* TEST INFRASTRUCTURE ONLY (oracle): drops the object-like macros that the reference's kernel
 * sources define (`#define width $WIDTH$`, ...) so the replay code after the include can use
 * those words as ordinary names again. */
#undef magnification
#undef sensitivity
#undef GxGyMagnification
#undef tSS
#undef tSO
#undef radius
#undef width
#undef height
#undef wh
#undef wInt
#undef hInt
#undef whInt
#undef wM
#undef hM
#undef whM
#undef whdM
#undef nFrameForSRRF
#undef intWeighting
#undef nPlanes
#undef dimRatio
#undef whd
#undef vxy_offset
#undef vxy_ArrayShift
