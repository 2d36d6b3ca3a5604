/* Minimal stand-ins for the MFC names that FEMM's fkn/spars.cpp touches, so the
 * reference's CPU sparse PCG (CBigLinProb) compiles unmodified with g++ for the
 * CPU baseline.  None of these do anything: the progress bar and message box
 * calls are no-ops. */
#pragma once
#include <cstdio>
typedef int BOOL;
#ifndef TRUE
#define TRUE 1
#define FALSE 0
#endif
#define IDC_FRAME1 1
#define IDC_FRAME2 2
struct CString {
  const char *text;
  CString(const char *t = "") : text(t) {}
  operator const char *() const { return text; }
};
struct CProgressCtrl {
  void SetPos(int) {}
};
template <typename... T> inline void MsgBox(const char *, T...) {}
