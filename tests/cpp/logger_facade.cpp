// The facade's UtilityLogger (no GPU needed): the message list keeps the last
// maxSize messages, quickLog formats printf-style, the level selects what
// getMsgListString returns, and each message is echoed as "sender>> text".
// Exits 0 on success.
#include <cstdio>
#include <string>

#include "behavert/BehaveRT.h"

using namespace BehaveRT;

int main() {
  UtilityLogger* log = m_CommonRes.getLogger();
  for (int i = 0; i < 60; ++i) log->quickLog("Flocking", "frame %d of %s", i, "demo");
  bool ok = log->getMsgList().size() == 50 && log->isModified();
  ok = ok && log->getMsgList().front().first.second == "frame 10 of demo";
  ok = ok && log->getMsgList().back().first.second == "frame 59 of demo";

  UtilityLogger small(3);
  small.log("A", "one");
  small.log("B", "two", UtilityLogger::LOG_DEBUG);
  small.log("A", "three");
  const std::string info = small.getMsgListString("|");   // info level: debug messages left out
  small.setLevelString("debug");
  const std::string all = small.getMsgListString("|");
  small.setSenderFilter("A");
  int fromA = 0;
  for (const UtilityLogger::logItem& item : small.getMsgList()) fromA += small.checkSender(item) ? 1 : 0;
  ok = ok && info == "one|three|" && all == "one|two|three|" && fromA == 2;
  std::printf("logger: %s\n", ok ? "yes" : "no");
  return ok ? 0 : 1;
}
