/* No-op stand-in for the FKN dialog: spars.cpp only reports progress through it. */
#pragma once
struct CFknDlg {
  CProgressCtrl m_prog1, m_prog2;
  void SetDlgItemText(int, const char *) {}
  void InvalidateRect(void *, int) {}
  void UpdateWindow() {}
};
