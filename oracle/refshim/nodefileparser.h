// nodefileparser.h stand-in (TEST INFRASTRUCTURE, see qshim.h): one host,
// one core, no GPU file.
#pragma once
#include "qshim.h"
namespace LangmuirCore {
class NodeFileParser {
public:
    QString hostName() { return QString("localhost"); }
    int numProc(const QString&) { return 1; }
    int GPUid(const QString&, int) { return -1; }
};
}  // namespace LangmuirCore
