// Test infrastructure only: an in-memory stand-in for the reference's
// SQLite-backed ProjectManager (ProjectManager.cpp needs sqlite3.c, which the
// reference tree does not ship), linked into oracle/_ref/libi360ref.so so that
// the reference's own StorageEngine (pixel-buffer framing and shard files),
// Tiff16Writer and PanoramaExporter run unmodified on files in a temporary
// directory.  Only the members those call are defined: the chunk grid of
// CreateProject (the rule of ProjectManager.cpp:260-281), the blob directory,
// and the STAGE3_RENDER tasks that ref_export_preview records.  No arithmetic
// of the reference is replaced.

#include "HeaderFiles/ProjectManager.h"

#include <string>
#include <vector>

namespace WindowsApp::Core
{
namespace
{
std::vector<BlobDirectoryEntry> g_blobs;
std::vector<Task> g_tasks;
}  // namespace

// Registers a completed render task of `chunkId` with output blob `blobId`.
void RefStubAddRenderTask(const std::string& chunkId, int64_t blobId)
{
    Task t;
    t.taskId = static_cast<int64_t>(g_tasks.size()) + 1;
    t.stage = PipelineStage::STAGE3_RENDER;
    t.unitKind = "chunk";
    t.unitKey = chunkId;
    t.status = TaskStatus::COMPLETED;
    t.outputBlobId = blobId;
    g_tasks.push_back(t);
}

ProjectManager::ProjectManager() = default;
ProjectManager::~ProjectManager() = default;

bool ProjectManager::CreateProject(const std::wstring& dbPath, int totalWidth, int totalHeight, int chunkSize)
{
    m_projectPath = dbPath;
    m_totalWidth = totalWidth;
    m_totalHeight = totalHeight;
    m_chunks.clear();
    g_blobs.clear();
    g_tasks.clear();
    for (int y = 0; y < totalHeight; y += chunkSize)
        for (int x = 0; x < totalWidth; x += chunkSize)
        {
            ChunkModel c;
            c.id = "C_" + std::to_string(x / chunkSize) + "_" + std::to_string(y / chunkSize);
            c.x_offset = x;
            c.y_offset = y;
            c.width = chunkSize < totalWidth - x ? chunkSize : totalWidth - x;
            c.height = chunkSize < totalHeight - y ? chunkSize : totalHeight - y;
            m_chunks.push_back(c);
        }
    return true;
}

void ProjectManager::CloseProject()
{
    m_chunks.clear();
    g_blobs.clear();
    g_tasks.clear();
}

int64_t ProjectManager::AddBlobDirectoryEntry(const BlobDirectoryEntry& entry)
{
    g_blobs.push_back(entry);
    g_blobs.back().blobId = static_cast<int64_t>(g_blobs.size());
    return g_blobs.back().blobId;
}

std::optional<BlobDirectoryEntry> ProjectManager::GetBlobDirectoryEntry(int64_t blobId) const
{
    if (blobId <= 0 || blobId > static_cast<int64_t>(g_blobs.size())) return std::nullopt;
    return g_blobs[static_cast<size_t>(blobId - 1)];
}

std::vector<Task> ProjectManager::GetTasksForStage(PipelineStage stage) const
{
    std::vector<Task> out;
    for (const auto& t : g_tasks)
        if (t.stage == stage) out.push_back(t);
    return out;
}
}  // namespace WindowsApp::Core
