/* Oracle build shim (test infrastructure only).
 * The reference's compute translation units name four VapourSynth types in
 * lgcr.h but never use their members; the oracle build only needs them to
 * exist. This is not the VapourSynth API header. */
#pragma once
struct VSNode;
struct VSPlugin;
struct VSPLUGINAPI;
struct VSVideoInfo { int placeholder; };
